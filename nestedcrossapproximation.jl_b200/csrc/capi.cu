// C ABI of the library (include/nca_b200.h): trees, partition, the device-resident batched
// build and the H^2 product. Host orchestration only; the arithmetic is in build_kernels.cu
// and apply_kernels.cu, the index planning in host_plan.cpp.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <chrono>
#include <cstring>
#include <exception>
#include <functional>
#include <future>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <type_traits>
#include <unordered_map>
#include <unordered_set>
#include <stdexcept>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include <sys/mman.h>

#include "apply_kernels.cuh"
#include "build_kernels.cuh"
#include "nca_internal.h"

namespace nca {

namespace {
thread_local std::string g_error;
thread_local int g_singular[4] = {0, 0, 0, 0};

struct Failure : std::runtime_error {
    int code;
    Failure(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void check(cudaError_t e, const char *what, int line) {
    if (e != cudaSuccess) {
        int code = e == cudaErrorMemoryAllocation ? NCA_ERR_OOM : NCA_ERR_CUDA;
        throw Failure(code, std::string("CUDA error in ") + what + " (capi.cu:" + std::to_string(line) +
                                "): " + cudaGetErrorString(e));
    }
}
#define CK(call) check((call), #call, __LINE__)

// Device blocks of the builds' large scratch (level buffers, transposed operators), kept for the
// process and handed to later builds instead of freed: cudaFree of a multi-GB block waits for the
// whole device and unmaps it (tens of ms at the end of every build, once 0.84 s). A request takes
// the smallest kept block of at least its size and at most twice it; blocks beyond kKeep bytes
// (NCA_SCRATCH_CACHE_GB, default 16) are freed when returned.
class DeviceCache {
  public:
    static DeviceCache &get() {
        static DeviceCache *cache = new DeviceCache;  // never destroyed: the driver frees at exit
        return *cache;
    }
    // a block of at least `bytes` on the current device
    void *acquire(size_t bytes) {
        int dev = 0;
        CK(cudaGetDevice(&dev));
        {
            std::lock_guard<std::mutex> g(mu_);
            std::multimap<size_t, void *> &fl = free_[dev];
            auto it = fl.lower_bound(bytes);
            if (it != fl.end() && it->first <= 2 * bytes) {
                void *q = it->second;
                kept_ -= it->first;
                fl.erase(it);
                return q;
            }
        }
        void *q = nullptr;
        CK(cudaMalloc(&q, bytes));
        std::lock_guard<std::mutex> g(mu_);
        block_[q] = Block{bytes, dev};
        return q;
    }
    // takes back a block of this cache (false: not one of its blocks)
    bool release(void *q) {
        {
            std::lock_guard<std::mutex> g(mu_);
            auto it = block_.find(q);
            if (it == block_.end()) return false;
            const Block b = it->second;
            if (kept_ + b.bytes <= keep_) {
                free_[b.device].emplace(b.bytes, q);
                kept_ += b.bytes;
                return true;
            }
            block_.erase(it);
        }
        cudaFree(q);
        return true;
    }

  private:
    struct Block {
        size_t bytes;
        int device;
    };
    DeviceCache() {
        const char *e = getenv("NCA_SCRATCH_CACHE_GB");
        keep_ = size_t((e ? std::max(0.0, atof(e)) : 16.0) * double(size_t(1) << 30));
    }
    std::mutex mu_;
    std::unordered_map<int, std::multimap<size_t, void *>> free_;  // kept blocks per device, by size
    std::unordered_map<void *, Block> block_;                        // every block the cache made
    size_t kept_ = 0, keep_ = 0;
};

template <typename T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    bool cached = false;  // from DeviceCache (alloc_scratch)
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p && !(cached && DeviceCache::get().release(p))) cudaFree(p);
        p = nullptr;
        n = 0;
        cached = false;
    }
    // build scratch: from the process's device cache, returned to it on release
    void alloc_scratch(size_t count) {
        release();
        n = count;
        p = static_cast<T *>(DeviceCache::get().acquire(sizeof(T) * std::max<size_t>(count, 1)));
        cached = true;
    }
    void alloc(size_t count) {
        release();
        n = count;
        CK(cudaMalloc(&p, sizeof(T) * std::max<size_t>(count, 1)));
    }
    // hands the array to `later` (freed by its owner once no stream needs it) instead of freeing
    // it now: cudaFree waits for the whole device, including other host threads' work
    void defer(std::vector<void *> &later) {
        if (p) later.push_back(p);
        p = nullptr;
        n = 0;
        cached = false;
    }
    void upload(const T *h, size_t count, cudaStream_t s) {
        alloc(count);
        if (count) CK(cudaMemcpyAsync(p, h, sizeof(T) * count, cudaMemcpyHostToDevice, s));
    }
    void upload(const std::vector<T> &v, cudaStream_t s) { upload(v.data(), v.size(), s); }
    void zero(cudaStream_t s) { CK(cudaMemsetAsync(p, 0, sizeof(T) * std::max<size_t>(n, 1), s)); }
    std::vector<T> download(cudaStream_t s) const {
        std::vector<T> h(n);
        if (n) CK(cudaMemcpyAsync(h.data(), p, sizeof(T) * n, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        return h;
    }
};

// uploads v into the scratch buffer b, reallocating only when b is too small (the old array
// goes to `later`)
template <typename T, typename A>
void upload_reuse(DBuf<T> &b, const std::vector<T, A> &v, cudaStream_t s, std::vector<void *> &later) {
    if (!b.p || v.size() > b.n) {
        b.defer(later);  // cudaFree here would wait for the work of every stream on the device
        b.alloc_scratch(v.size());
    }
    if (!v.empty()) CK(cudaMemcpyAsync(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
}

// page-locked host array (downloads that need no staging copy)
template <typename T>
struct PinnedBuf {
    T *p = nullptr;
    explicit PinnedBuf(size_t n) { CK(cudaMallocHost(&p, sizeof(T) * std::max<size_t>(n, 1))); }
    PinnedBuf(const PinnedBuf &) = delete;
    PinnedBuf &operator=(const PinnedBuf &) = delete;
    ~PinnedBuf() {
        if (p) cudaFreeHost(p);
    }
    // hands the array to `later` instead of freeing it now (cudaFreeHost waits for the device)
    void defer(std::vector<void *> &later) {
        if (p) later.push_back(p);
        p = nullptr;
    }
};

// Page-locked staging blocks for the builds' plan uploads, kept for the process and handed out
// to the threads of later builds (uploads from pageable vectors go through the driver's staging
// at a few GB/s and serialise across threads; from page-locked memory they are DMA copies).
// Blocks beyond kPinnedKeep bytes in total are freed when returned.
class PinnedPool {
  public:
    struct Block {
        unsigned char *p = nullptr;
        size_t n = 0;
    };
    static PinnedPool &get() {
        static PinnedPool pool;
        return pool;
    }
    Block acquire(size_t n) {
        {
            std::lock_guard<std::mutex> g(mu_);
            size_t best = free_.size();
            for (size_t i = 0; i < free_.size(); ++i)
                if (free_[i].n >= n && (best == free_.size() || free_[i].n < free_[best].n)) best = i;
            if (best < free_.size()) {
                const Block b = free_[best];
                free_.erase(free_.begin() + long(best));
                kept_ -= b.n;
                return b;
            }
        }
        Block b;
        b.n = std::max<size_t>((n + (size_t(64) << 20) - 1) & ~((size_t(64) << 20) - 1), size_t(64) << 20);
        if (cudaHostAlloc(reinterpret_cast<void **>(&b.p), b.n, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            b.p = nullptr;
            b.n = 0;
        }
        return b;
    }
    void release(Block b) {
        if (!b.p) return;
        std::lock_guard<std::mutex> g(mu_);
        if (kept_ + b.n > kPinnedKeep) {
            cudaFreeHost(b.p);
            return;
        }
        kept_ += b.n;
        free_.push_back(b);
    }

  private:
    static constexpr size_t kPinnedKeep = size_t(2) << 30;
    std::mutex mu_;
    std::vector<Block> free_;
    size_t kept_ = 0;
};

// Host blocks for the builds' large transient arrays (gather plan lists and records), kept for
// the process and handed to the threads of later builds. A fresh page costs a fault and a zero
// fill on first touch: on the build host, 8 threads each filling 96 MB of fresh memory took 63-67
// ms against 15 ms for memory already mapped. Blocks are sized in powers of two from 2 MiB and
// kept on free lists by size, up to kHostKeep bytes; smaller requests go to operator new. (No
// huge-page advice: with the hosts' defrag=madvise setting a fault in an advised range may stall
// on memory compaction, and the driver's own mappings wait behind it.)
class HostPool {
  public:
    static constexpr size_t kMin = size_t(2) << 20;
    static HostPool &get() {
        static HostPool *pool = new HostPool;  // never destroyed: blocks may outlive static teardown
        return *pool;
    }
    static size_t block_size(size_t bytes) {
        size_t c = kMin;
        while (c < bytes) c <<= 1;
        return c;
    }
    void *acquire(size_t cap) {
        {
            std::lock_guard<std::mutex> g(mu_);
            auto it = free_.find(cap);
            if (it != free_.end() && !it->second.empty()) {
                void *p = it->second.back();
                it->second.pop_back();
                kept_ -= cap;
                return p;
            }
        }
        void *p = mmap(nullptr, cap, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
        if (p == MAP_FAILED) throw std::bad_alloc();
        return p;
    }
    void release(void *p, size_t cap) {
        {
            std::lock_guard<std::mutex> g(mu_);
            if (kept_ + cap <= kHostKeep) {
                free_[cap].push_back(p);
                kept_ += cap;
                return;
            }
        }
        munmap(p, cap);
    }

  private:
    static constexpr size_t kHostKeep = size_t(4) << 30;
    std::mutex mu_;
    std::unordered_map<size_t, std::vector<void *>> free_;
    size_t kept_ = 0;
};

// std::vector allocator over HostPool for arrays of 2 MiB and more
template <typename T>
struct PoolAlloc {
    using value_type = T;
    PoolAlloc() = default;
    template <typename U>
    PoolAlloc(const PoolAlloc<U> &) {}
    T *allocate(size_t n) {
        const size_t bytes = n * sizeof(T);
        if (bytes < HostPool::kMin) return static_cast<T *>(::operator new(bytes));
        return static_cast<T *>(HostPool::get().acquire(HostPool::block_size(bytes)));
    }
    void deallocate(T *p, size_t n) {
        const size_t bytes = n * sizeof(T);
        if (bytes < HostPool::kMin) {
            ::operator delete(p);
            return;
        }
        HostPool::get().release(p, HostPool::block_size(bytes));
    }
    template <typename U>
    bool operator==(const PoolAlloc<U> &) const {
        return true;
    }
    template <typename U>
    bool operator!=(const PoolAlloc<U> &) const {
        return false;
    }
};
template <typename T>
using hvec = std::vector<T, PoolAlloc<T>>;

// Uploads through one page-locked block (pageable copies when no block could be had); the block
// goes back to the pool once the stream has finished the copies.
class StagedUploads {
  public:
    // bytes: the most the staged arrays need; the block is taken at the first staged array
    StagedUploads(size_t bytes, cudaStream_t s) : s_(s), want_(bytes + 256) {}
    ~StagedUploads() {
        flush();
        if (b_.p) {
            cudaStreamSynchronize(s_);  // the block is not reused before its copies
            PinnedPool::get().release(b_);
        }
    }
    // allocates d and queues its upload: the copies are issued by flush() (or the destructor), so
    // the sources must live until then and no kernel may read d before it
    template <typename T, typename A>
    void up(DBuf<T> &d, const std::vector<T, A> &v) {
        d.alloc(v.size());
        if (v.empty()) return;
        const size_t bytes = sizeof(T) * v.size();
        if (!b_.p && !tried_) {
            b_ = PinnedPool::get().acquire(want_);
            tried_ = true;
        }
        used_ = (used_ + 15) & ~size_t(15);
        if (b_.p && used_ + bytes <= b_.n) {
            jobs_.push_back(Job{d.p, v.data(), bytes, used_});
            used_ += bytes;
        } else {
            CK(cudaMemcpyAsync(d.p, v.data(), bytes, cudaMemcpyHostToDevice, s_));
        }
    }
    // the queued arrays into the page-locked block (each array on a thread of its own when they
    // are large: a plan's ~100 MB took ~10 ms on one), then one DMA copy each
    void flush() {
        if (jobs_.empty()) return;
        size_t total = 0;
        for (const Job &j : jobs_) total += j.bytes;
        auto stage = [&](const Job &j) { std::memcpy(b_.p + j.at, j.src, j.bytes); };
        if (total < (size_t(8) << 20) || jobs_.size() == 1) {
            for (const Job &j : jobs_) stage(j);
        } else {
            std::vector<std::thread> pool;
            for (size_t k = 1; k < jobs_.size(); ++k) pool.emplace_back(stage, std::cref(jobs_[k]));
            stage(jobs_[0]);
            for (auto &th : pool) th.join();
        }
        for (const Job &j : jobs_) CK(cudaMemcpyAsync(j.dst, b_.p + j.at, j.bytes, cudaMemcpyHostToDevice, s_));
        jobs_.clear();
    }
    StagedUploads(const StagedUploads &) = delete;
    StagedUploads &operator=(const StagedUploads &) = delete;

  private:
    struct Job {
        void *dst;
        const void *src;
        size_t bytes, at;
    };
    cudaStream_t s_;
    size_t want_;
    PinnedPool::Block b_;
    bool tried_ = false;
    size_t used_ = 0;
    std::vector<Job> jobs_;
};

template <typename T>
std::vector<T> download_now(const DBuf<T> &b, size_t n) {
    std::vector<T> h(n);
    if (n) CK(cudaMemcpy(h.data(), b.p, sizeof(T) * n, cudaMemcpyDeviceToHost));
    return h;
}

int fail(int code, const std::string &msg) {
    g_error = msg;
    return code;
}

template <typename F>
int guarded(F &&f) {
    try {
        return f();
    } catch (const Failure &e) {
        return fail(e.code, e.what());
    } catch (const std::bad_alloc &) {
        return fail(NCA_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(NCA_ERR_ARG, e.what());
    }
}

// Node lists grouped by level: nodes[ptr[l] .. ptr[l+1]) for level order as listed.
struct LevelLists {
    std::vector<int32_t> ptr, nodes;
    std::vector<int> mcap;  // per group: capacity (rows) used for shared memory
    DBuf<int32_t> d_nodes;
};

}  // namespace

void set_error(const std::string &msg) { g_error = msg; }
void set_singular(int side, int node, int npivots, int rank) {
    g_singular[0] = side;
    g_singular[1] = node;
    g_singular[2] = npivots;
    g_singular[3] = rank;
}

}  // namespace nca

using namespace nca;

struct DevSide {
    int nnodes = 0, nlevels = 0;
    int64_t npts = 0;
    DBuf<double> pts;
    DBuf<int32_t> perm, begin, end, firstchild, nchildren;
    DBuf<int32_t> fpptr, fpidx;
    DBuf<int32_t> rank, nrows, piv;
    DBuf<int64_t> xoff, cptr;
    DBuf<double2> X, XT;  // interpolation operators and their transposes (same padded offsets)
    DBuf<float2> X32, XT32;
    DBuf<int32_t> cpiv;     // column pivots sigma of every node (far-side point ids, maxrank per node)
    DBuf<double2> dX, dXT;  // dX/dk on the frozen skeleton (prepared on demand)
    std::vector<int32_t> h_fpptr, h_fpidx, h_rank, h_nrows, h_piv;
    std::vector<int64_t> h_xoff, h_cptr;
    LevelLists up, down;
    DBuf<int32_t> leaves;
    int nleaves = 0, leafcap = 0;
};

// ---- directional cores: basis items (one per (cluster, direction)) and gather plans ----
struct DirItems {
    nca::DirSide plan;
    int nitems = 0;
    std::vector<int32_t> h_rank, h_nrows;  // item pivots stay on the device
    std::vector<int64_t> h_xoff, h_cptr;
    DBuf<int32_t> item_node, item_basis, item_chptr, item_chidx, rank, nrows, piv;
    DBuf<int32_t> cpiv;  // column pivots sigma of every item (maxrank per item): frozen-skeleton refills
    DBuf<int64_t> xoff;
    DBuf<double2> X, XT;
    // device and page-locked scratch of the build, freed once the build has synchronised
    std::vector<void *> later, later_host;
    void free_later() {
        for (void *q : later)
            if (!DeviceCache::get().release(q)) cudaFree(q);
        for (void *q : later_host) cudaFreeHost(q);
        later.clear();
        later_host.clear();
    }
    ~DirItems() { free_later(); }
};

// One product stage as block-sparse gathers over the vector arena: outputs (ordered by launch
// group), their segments, and the stage's block store.
struct GatherStage {
    std::vector<int32_t> group_ptr;  // launch groups (levels) over the outputs
    std::vector<int> group_maxrows;
    std::vector<double> group_work;  // mean block entries per output of each group
    DBuf<int32_t> outputs, rows, segptr, w;
    DBuf<int64_t> out, moff, voff;
    DBuf<WideOut> wout;  // the outputs in launch order as records (all-column FP32 gathers)
    DBuf<WideOut> tout;  // every output as a record, in group order (tensor-core gathers)
    // launches of the all-column FP32 kernel: group g's are [wide_gptr[g], wide_gptr[g + 1]), each
    // wide_count outputs from position wide_begin with the register tile wide_nr
    std::vector<int32_t> wide_gptr, wide_begin, wide_count;
    std::vector<int> wide_nr;
    DBuf<double2> M;
    DBuf<float2> M32;
    DBuf<double2> dM;     // d/dk of the store (frozen skeleton), prepared on demand
    int64_t entries = 0;  // algorithmic entries of the store
    // the copies that fill M from the side's operators (kept for refills at another wavenumber)
    DBuf<int64_t> c_soff, c_doff;
    DBuf<int32_t> c_ld, c_rows, c_cols;
    int64_t ncopies = 0;
};

// Products of one orientation: mode N (test <- trial) or T (trial <- test; C conjugates it).
// Arena rows: [0, nin) gathered x, [nin, nin + cin) input-side coefficients, then output-side.
struct DirProduct {
    int64_t nin = 0, nout = 0, cin = 0, cout = 0;
    GatherStage up, couple, down, leaves;
    // a mirrored Galerkin core (both sides one skeleton): the transposed product's up, down and
    // leaf stages are the forward product's (the same plans over the same stores); `same` points
    // at that product and this product's own three stay empty
    DirProduct *same = nullptr;
    bool same_couple = false;  // ... and the coupling stage too (the transposed blocks are the blocks)
    GatherStage &up_stage() { return same ? same->up : up; }
    GatherStage &couple_stage() { return same && same_couple ? same->couple : couple; }
    GatherStage &down_stage() { return same ? same->down : down; }
    GatherStage &leaf_stage() { return same ? same->leaves : leaves; }
    // the stages this product owns (the shared ones belong to `same`)
    std::vector<GatherStage *> own_stages() {
        if (same) return same_couple ? std::vector<GatherStage *>{} : std::vector<GatherStage *>{&couple};
        return {&up, &couple, &down, &leaves};
    }
};

struct DirCore {
    DirItems side[2];
    DirProduct prod[2];
    // coupling blocks S_e = K[tau_t, tau_s] per far pair (test order) and their transposition plan
    DBuf<int32_t> cpair_it, cpair_is, ctr_rows, ctr_cols;
    DBuf<int64_t> ccoff, ctr_in, ctr_off;
    int64_t npairs = 0, ntr = 0;
};

struct nca_core {
    int device = 0;
    int maxrank = 50;
    bool f32 = false;
    nca::Tree tree[2];
    nca::Partition part;
    KernelParams K{};
    DBuf<double2> kmat;
    DevSide side[2];
    // couplings in test-node CSR order
    DBuf<int32_t> farptr, farnodes, tfarptr, tfarnodes, tfarpair;
    // padded block offsets: S_ts per test-CSR pair (cfoff), S_ts^T per trial-CSR entry (ctoff)
    DBuf<int64_t> cfoff, ctoff;
    DBuf<double2> C, CT;
    DBuf<float2> C32, CT32;
    std::vector<int64_t> h_cfoff;
    DBuf<int32_t> couple_fwd, couple_rev;
    int n_couple_fwd = 0, n_couple_rev = 0;
    // near field: one row block per test node
    DBuf<int32_t> nearptr, nearnodes, tnearptr, tnearnodes;
    // padded block offsets: N_ts per test-CSR near pair (nfoff), N_ts^T per trial-CSR entry (ntoff)
    DBuf<int64_t> nfoff, ntoff;
    DBuf<double2> N, NT;
    DBuf<float2> N32, NT32;
    std::vector<int64_t> h_nfoff;
    std::vector<int64_t> h_noff;  // compact row-block offsets per test node (exports)
    std::vector<int32_t> h_ncols;
    // pair lists and transposition plans of the coupling and near stores (refills at another
    // wavenumber and the d/dk stores reuse them)
    DBuf<int32_t> cpair_t, ctr_rows, ctr_cols, near_t, ntr_rows, ntr_cols;
    DBuf<int64_t> ctr_in, ntr_in;
    int64_t n_ctr = 0, n_ntr = 0;
    DBuf<double2> dC, dCT, dN, dNT;  // dS/dk and dN/dk on the frozen skeleton
    bool has_dk = false;
    bool batch = false;  // block-diagonal batch of several cores (one wavenumber per member)
    std::unique_ptr<DirCore> dir;  // directional (wideband) core: items and gather plans
    nca::Wideband wb{};            // the wideband admissibility of a directional core
    nca_core_info info{};
    bool moved = false;  // stores moved into a batch: the core may only be destroyed
};

struct nca_workspace {
    nca_core *core = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int max_nrhs = 0;
    DBuf<double2> xt, xhat, yhat, xstage, ystage;
    DBuf<double2> dxhat, dyhat;  // tangent products (d/dk)
    DBuf<double2> arena;         // directional products: [x; input coefficients; output coefficients]
    std::atomic<bool> busy{false};
    DBuf<int32_t> error;
    int32_t *error_host = nullptr;  // pinned
    double last_seconds = 0.0;
    int last_launches = 0;
    bool far = true, near = true;
    bool profiling = false;
    cudaEvent_t stage_ev[9] = {};  // StageEvent order
    // directional products: an event pair around every stage of every 16-column pass (grown on
    // demand) and the stage of each pair
    std::vector<cudaEvent_t> dir_ev;
    std::vector<int> dir_stage;
    double stage_seconds[6] = {0, 0, 0, 0, 0, 0};
    int stage_launches[6] = {0, 0, 0, 0, 0, 0};
    // far-field sweeps beside the near field: a second stream (higher priority, so the sweeps'
    // small launches take SM slots as the near-field CTAs retire) and its fork / join events
    cudaStream_t aux = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    int aux_priority = 0;
    // Products repeated with identical arguments on device arrays replay a CUDA graph of their
    // launches: a call whose arguments were seen in one of the last few calls is captured once,
    // later identical calls launch the graph. Buffer reallocation (gen) invalidates every graph.
    struct GraphKey {
        int mode, precision, b, far, near, profiling, overlap;
        const void *x, *y;
        int64_t ldx, ldy;
        double ar, ai, br, bi;
        uint64_t gen;
        bool operator==(const GraphKey &o) const {
            return mode == o.mode && precision == o.precision && b == o.b && far == o.far && near == o.near &&
                   profiling == o.profiling && overlap == o.overlap && x == o.x && y == o.y && ldx == o.ldx &&
                   ldy == o.ldy && ar == o.ar &&
                   ai == o.ai && br == o.br && bi == o.bi && gen == o.gen;
        }
    };
    struct Graph {
        GraphKey key;
        cudaGraphExec_t exec = nullptr;
        int launches = 0;
        int stage[6] = {0, 0, 0, 0, 0, 0};
    };
    std::vector<Graph> graphs;     // at most kGraphs, oldest first
    std::vector<GraphKey> seen;    // the last few eager calls' arguments
    uint64_t gen = 0;
    bool use_graphs = false;
    bool use_overlap = true;  // near field beside the sweeps (second stream)
};

namespace {

constexpr size_t kGraphs = 4;

constexpr int kMaxSmem = 227 * 1024;

// Block sizes rounded up to an even number of entries: every block then starts on a 32-byte
// (FP64) or 16-byte (FP32) boundary, as the bulk copies of the product require.
inline int64_t pad2(int64_t n) { return (n + 1) & ~int64_t(1); }
// Row slots of a vector buffer that serves every b' <= b right-hand sides: vector_stride(b') is
// b' plus at most 3 padding slots.
inline int vector_slots(int b) { return b + 3; }

void set_kernel_params(nca_core *c, const nca_kernel_desc *k, int64_t ntest, int64_t ntrial,
                       cudaStream_t s) {
    c->K.kind = k->kind;
    c->K.sign = k->sign < 0 ? -1 : 1;
    c->K.k = k->k;
    c->K.rmin = k->rmin;
    c->K.mat = nullptr;
    c->K.ldmat = 0;
    if (k->kind == NCA_KERNEL_MATRIX) {
        if (!k->matrix || k->ldmatrix < ntest) throw Failure(NCA_ERR_ARG, "matrix kernel needs ldmatrix >= ntest");
        c->kmat.upload(reinterpret_cast<const double2 *>(k->matrix), size_t(k->ldmatrix) * ntrial, s);
        c->K.mat = c->kmat.p;
        c->K.ldmat = k->ldmatrix;
    } else if (k->kind != NCA_KERNEL_HELMHOLTZ && k->kind != NCA_KERNEL_LAPLACE) {
        throw Failure(NCA_ERR_ARG, "unknown kernel kind");
    }
}

void upload_tree(DevSide &d, const nca::Tree &T, const double *pts, cudaStream_t s) {
    d.nnodes = T.nnodes;
    d.nlevels = T.nlevels;
    d.npts = T.npoints;
    d.pts.upload(pts, size_t(3 * T.npoints), s);
    d.perm.upload(T.perm, s);
    d.begin.upload(T.begin, s);
    d.end.upload(T.end, s);
    d.firstchild.upload(T.firstchild, s);
    d.nchildren.upload(T.nchildren, s);
}

// CSR of n lists filled by fill(i, list) on the host's worker threads (contiguous item ranges
// per thread, concatenated in item order).
template <typename F, typename PV, typename IV>
void parallel_csr(int n, F fill, PV &ptr, IV &idx) {
    // a thread per 2,048 lists at least: short lists (the deepest levels) are not worth a pool
    const int nth = std::max(1, std::min(nca::host_threads(), (n + 2047) / 2048));
    std::vector<hvec<int64_t>> lptr(nth);  // pooled: the lists are rebuilt level by level
    std::vector<hvec<int32_t>> lidx(nth);
    auto work = [&](int w) {
        const int i0 = int(int64_t(n) * w / nth), i1 = int(int64_t(n) * (w + 1) / nth);
        std::vector<int32_t> one;
        lptr[w].assign(1, 0);
        for (int i = i0; i < i1; ++i) {
            fill(i, one);
            lidx[w].insert(lidx[w].end(), one.begin(), one.end());
            lptr[w].push_back(int64_t(lidx[w].size()));
        }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < nth; ++w) pool.emplace_back(work, w);
    work(0);
    for (auto &th : pool) th.join();
    // the threads' pieces back to back, each copied by its own thread
    std::vector<int64_t> off(nth + 1, 0);
    for (int w = 0; w < nth; ++w) off[w + 1] = off[w] + int64_t(lidx[w].size());
    ptr.assign(size_t(n) + 1, 0);
    idx.resize(size_t(off[nth]));
    auto place = [&](int w) {
        const int i0 = int(int64_t(n) * w / nth);
        for (size_t k = 1; k < lptr[w].size(); ++k) ptr[size_t(i0) + k] = lptr[w][k] + off[w];
        std::copy(lidx[w].begin(), lidx[w].end(), idx.begin() + off[w]);
        hvec<int32_t>().swap(lidx[w]);
    };
    pool.clear();
    for (int w = 1; w < nth; ++w) pool.emplace_back(place, w);
    place(0);
    for (auto &th : pool) th.join();
}

// Centroids of every cluster of a tree (the host planner's sums, in its order), on the host threads.
std::vector<double> cluster_centroids(const nca::Tree &own, const double *ownpts) {
    std::vector<double> centroid(3 * size_t(own.nnodes), 0.0);
    std::atomic<int> cursor{0};
    auto work = [&]() {
        for (;;) {
            const int t = cursor.fetch_add(1);
            if (t >= own.nnodes) break;
            if (own.size(t) > 0)
                nca::cluster_centroid(ownpts, own.perm.data() + own.begin[t], own.size(t), &centroid[3 * size_t(t)]);
        }
    };
    const int nth = std::max(1, std::min(nca::host_threads(), own.nnodes));
    std::vector<std::thread> pool;
    for (int i = 1; i < nth; ++i) pool.emplace_back(work);
    work();
    for (auto &th : pool) th.join();
    return centroid;
}

// Phase 1 on the device: tree-mimicry far pivots of every item of one side (item i is own
// cluster item_node[i], or cluster i when item_node is null), with far field ffnodes[ffptr[i]..)
// in the reference's farfield order. Returns the CSR of pivots (far point ids) on the device
// (dptr, didx) and its pointer array on the host; the host copy of the list only when asked for.
void device_farpivots(const nca::Tree &own, const double *ownpts, const nca::Tree &far, const DevSide &fd,
                      int nitems, const std::vector<int64_t> &ffptr, const std::vector<int32_t> &ffnodes,
                      const std::vector<int32_t> *item_node, int maxrank, cudaStream_t s,
                      std::vector<int32_t> &fpptr, DBuf<int32_t> &dfpptr, DBuf<int32_t> &dfpidx,
                      std::vector<int32_t> *fpidx) {
    fpptr.assign(nitems + 1, 0);
    if (fpidx) fpidx->clear();
    if (nitems == 0) {
        dfpptr.upload(fpptr, s);
        dfpidx.alloc(1);
        return;
    }
    const std::vector<double> centroid = cluster_centroids(own, ownpts);
    std::vector<int32_t> own_size(own.nnodes);
    for (int t = 0; t < own.nnodes; ++t) own_size[t] = own.size(t);
    DBuf<int64_t> dptr;
    DBuf<int32_t> dnodes, ditem, dsize, dcount, dpiv, derr;
    DBuf<double> dcent, dcenter;
    dptr.upload(ffptr, s);
    dnodes.upload(ffnodes, s);
    if (item_node) ditem.upload(*item_node, s);
    dsize.upload(own_size, s);
    dcent.upload(centroid, s);
    dcenter.upload(far.center, s);
    dcount.alloc(nitems);
    dpiv.alloc(size_t(nitems) * maxrank);
    derr.alloc(2);  // error word, item cursor
    derr.zero(s);
    MimicryArgs a{};
    a.begin = fd.begin.p;
    a.end = fd.end.p;
    a.firstchild = fd.firstchild.p;
    a.nchildren = fd.nchildren.p;
    a.perm = fd.perm.p;
    a.center = dcenter.p;
    a.pts = fd.pts.p;
    a.nitems = nitems;
    a.ffptr = dptr.p;
    a.ffnodes = dnodes.p;
    a.item_node = item_node ? ditem.p : nullptr;
    a.centroid = dcent.p;
    a.own_size = dsize.p;
    a.maxrank = maxrank;
    a.count = dcount.p;
    a.piv = dpiv.p;
    a.error = derr.p;
    a.cursor = derr.p + 1;
    launch_mimicry(a, s);
    CK(cudaGetLastError());
    const std::vector<int32_t> count = dcount.download(s);
    const std::vector<int32_t> err = derr.download(s);
    if (err[0] != 0) throw Failure(NCA_ERR_CUDA, "internal: tree mimicry ran out of far points");
    for (int i = 0; i < nitems; ++i) fpptr[i + 1] = fpptr[i] + count[i];
    dfpptr.upload(fpptr, s);
    dfpidx.alloc(size_t(std::max(fpptr[nitems], 1)));
    launch_compact_pivots(dpiv.p, maxrank, dcount.p, dfpptr.p, nitems, dfpidx.p, s);
    CK(cudaGetLastError());
    if (fpidx) {
        fpidx->resize(fpptr[nitems]);
        if (fpptr[nitems])
            CK(cudaMemcpyAsync(fpidx->data(), dfpidx.p, sizeof(int32_t) * fpptr[nitems], cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
}

// Rows/rank bounds per node (bottom-up), X slot offsets and per-level active node lists.
void plan_side(DevSide &d, const nca::Tree &T, int maxrank, std::vector<int32_t> &lv_ptr,
               std::vector<int32_t> &lv_nodes, std::vector<int> &lv_mcap, std::vector<int> &lv_ncap) {
    std::vector<int64_t> mb(T.nnodes, 0), rb(T.nnodes, 0);
    for (int node = T.nnodes - 1; node >= 0; --node) {
        int nfp = d.h_fpptr[node + 1] - d.h_fpptr[node];
        if (nfp == 0) continue;
        int64_t m = 0;
        if (T.isleaf(node)) {
            m = T.size(node);
        } else {
            for (int c = 0; c < T.nchildren[node]; ++c) m += rb[T.firstchild[node] + c];
        }
        mb[node] = m;
        rb[node] = std::min<int64_t>({int64_t(maxrank), m, int64_t(nfp)});
    }
    d.h_xoff.assign(T.nnodes + 1, 0);
    for (int node = 0; node < T.nnodes; ++node) d.h_xoff[node + 1] = d.h_xoff[node] + pad2(mb[node] * rb[node]);
    lv_ptr.assign(1, 0);
    lv_nodes.clear();
    lv_mcap.clear();
    lv_ncap.clear();
    for (int lev = T.nlevels - 1; lev >= 0; --lev) {
        int mc = 0, nc = 0;
        for (int node = T.levelptr[lev]; node < T.levelptr[lev + 1]; ++node) {
            int nfp = d.h_fpptr[node + 1] - d.h_fpptr[node];
            if (nfp == 0) continue;
            lv_nodes.push_back(node);
            mc = std::max<int>(mc, int(mb[node]));
            nc = std::max(nc, nfp);
        }
        lv_ptr.push_back(int32_t(lv_nodes.size()));
        lv_mcap.push_back(mc);
        lv_ncap.push_back(nc);
    }
}

// Apply plans of one side once the ranks are known.
void plan_apply(DevSide &d, const nca::Tree &T, cudaStream_t s) {
    d.up.ptr.assign(1, 0);
    d.up.nodes.clear();
    d.up.mcap.clear();
    for (int lev = T.nlevels - 1; lev >= 0; --lev) {
        int mc = 0;
        for (int node = T.levelptr[lev]; node < T.levelptr[lev + 1]; ++node)
            if (d.h_rank[node] > 0) {
                d.up.nodes.push_back(node);
                mc = std::max(mc, d.h_rank[node]);
            }
        d.up.ptr.push_back(int32_t(d.up.nodes.size()));
        d.up.mcap.push_back(mc);
    }
    d.up.d_nodes.upload(d.up.nodes, s);
    d.down.ptr.assign(1, 0);
    d.down.nodes.clear();
    d.down.mcap.clear();
    for (int lev = 0; lev < T.nlevels; ++lev) {
        int mc = 0;
        for (int node = T.levelptr[lev]; node < T.levelptr[lev + 1]; ++node)
            if (d.h_rank[node] > 0 && !T.isleaf(node)) {
                d.down.nodes.push_back(node);
                mc = std::max(mc, d.h_nrows[node]);
            }
        d.down.ptr.push_back(int32_t(d.down.nodes.size()));
        d.down.mcap.push_back(mc);
    }
    d.down.d_nodes.upload(d.down.nodes, s);
    std::vector<int32_t> leaves;
    d.leafcap = 0;
    for (int node = 0; node < T.nnodes; ++node)
        if (T.isleaf(node)) {
            leaves.push_back(node);
            d.leafcap = std::max(d.leafcap, T.size(node));
        }
    d.nleaves = int(leaves.size());
    d.leaves.upload(leaves, s);
    d.h_cptr.assign(T.nnodes + 1, 0);
    for (int node = 0; node < T.nnodes; ++node) d.h_cptr[node + 1] = d.h_cptr[node] + d.h_rank[node];
    d.cptr.upload(d.h_cptr, s);
}

int launch_grid(int64_t work, int per_sm) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return int(std::max<int64_t>(1, std::min<int64_t>(work, int64_t(sms) * per_sm)));
}

// Couplings S_ts = K[tau_t, tau_s] of every admissible pair (test CSR order) into C and their
// transposes (trial CSR order) into CT, for the kernel K (values or d/dk entries).
void fill_couplings(nca_core *c, const KernelParams &K, double2 *C, double2 *CT, cudaStream_t s) {
    const int64_t npairs = int64_t(c->part.farnodes.size());
    CouplingArgs a;
    a.K = K;
    a.test_pts = c->side[0].pts.p;
    a.trial_pts = c->side[1].pts.p;
    a.pair_t = c->cpair_t.p;
    a.pair_s = c->farnodes.p;
    a.rank_t = c->side[0].rank.p;
    a.rank_s = c->side[1].rank.p;
    a.piv_t = c->side[0].piv.p;
    a.piv_s = c->side[1].piv.p;
    a.maxrank = c->maxrank;
    a.coff = c->cfoff.p;
    a.npairs = npairs;
    a.C = C;
    a.C32 = nullptr;
    if (npairs > 0) {
        k_couplings<<<launch_grid(npairs, 16), 256, 0, s>>>(a);
        CK(cudaGetLastError());
    }
    launch_transpose_blocks<double2>(C, c->ctr_in.p, c->ctr_rows.p, c->ctr_cols.p, c->ctoff.p, c->n_ctr, CT, s);
    CK(cudaGetLastError());
}

// Near blocks K[t, s] of every near pair (test CSR order) into N and their transposes into NT.
void fill_near(nca_core *c, const KernelParams &K, double2 *N, double2 *NT, cudaStream_t s) {
    const int64_t nnear = int64_t(c->part.nearnodes.size());
    NearArgs a;
    a.K = K;
    a.test_pts = c->side[0].pts.p;
    a.trial_pts = c->side[1].pts.p;
    a.pair_t = c->near_t.p;
    a.pair_s = c->nearnodes.p;
    a.t_perm = c->side[0].perm.p;
    a.t_begin = c->side[0].begin.p;
    a.t_end = c->side[0].end.p;
    a.s_perm = c->side[1].perm.p;
    a.s_begin = c->side[1].begin.p;
    a.s_end = c->side[1].end.p;
    a.poff = c->nfoff.p;
    a.npairs = nnear;
    a.N = N;
    if (nnear > 0) {
        k_near<<<launch_grid(nnear, 16), 256, 0, s>>>(a);
        CK(cudaGetLastError());
    }
    launch_transpose_blocks<double2>(N, c->ntr_in.p, c->ntr_rows.p, c->ntr_cols.p, c->ntoff.p, c->n_ntr, NT, s);
    CK(cudaGetLastError());
}

// Complex FP32 copies of every store (the mixed-precision product reads them).
void make_f32_copies(nca_core *c, cudaStream_t s) {
    auto down = [&](DBuf<double2> &src, DBuf<float2> &dst) {
        if (dst.n != src.n) dst.alloc(src.n);
        if (src.n) k_to_f32<<<launch_grid(int64_t(src.n) / 256 + 1, 8), 256, 0, s>>>(src.p, dst.p, int64_t(src.n));
        CK(cudaGetLastError());
    };
    for (int sd = 0; sd < 2; ++sd) {
        down(c->side[sd].X, c->side[sd].X32);
        down(c->side[sd].XT, c->side[sd].XT32);
    }
    down(c->C, c->C32);
    down(c->CT, c->CT32);
    down(c->N, c->N32);
    down(c->NT, c->NT32);
}

// Interpolation operators of one side on the frozen skeleton (k_level_values): mode 0 the values
// for kernel K into Xout, mode 1 dX/dk (dK: derivative entries) from the side's X; transposes
// into XTout. A singular cross matrix raises NCA_ERR_SINGULAR and leaves Xout partly written.
void fill_bases(nca_core *c, int sd, int mode, const KernelParams &K, const KernelParams &dK, double2 *Xout,
                double2 *XTout, cudaStream_t s) {
    DevSide &d = c->side[sd];
    if (d.up.nodes.empty()) return;
    int mcap = 1, rcap = 1;
    for (int node = 0; node < d.nnodes; ++node)
        if (d.h_rank[node] > 0) {
            mcap = std::max(mcap, d.h_nrows[node]);
            rcap = std::max(rcap, d.h_rank[node]);
        }
    const size_t sm = values_smem_bytes(mcap, rcap, mode);
    if (sm > size_t(kMaxSmem))
        throw Failure(NCA_ERR_ARG, "a cross block of the frozen skeleton does not fit in shared memory");
    CK(cudaFuncSetAttribute(k_level_values, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    DBuf<int32_t> status;
    status.alloc(4);
    status.zero(s);
    ValueArgs a{};
    a.K = K;
    a.dK = dK;
    a.side = sd;
    a.mode = mode;
    a.own_pts = d.pts.p;
    a.far_pts = c->side[1 - sd].pts.p;
    a.perm = d.perm.p;
    a.begin = d.begin.p;
    a.end = d.end.p;
    a.firstchild = d.firstchild.p;
    a.nchildren = d.nchildren.p;
    a.rank = d.rank.p;
    a.piv = d.piv.p;
    a.cpiv = d.cpiv.p;
    a.maxrank = c->maxrank;
    a.Xin = d.X.p;
    a.Xout = Xout;
    a.xoff = d.xoff.p;
    a.status = status.p;
    k_level_values<<<int(d.up.nodes.size()), 256, sm, s>>>(a, d.up.d_nodes.p, mcap, rcap);
    CK(cudaGetLastError());
    const std::vector<int32_t> st = status.download(s);
    CK(cudaStreamSynchronize(s));
    if (st[0] == 1) {
        set_singular(sd, st[1], st[2], st[3]);
        throw Failure(NCA_ERR_SINGULAR, "SingularCrossMatrixError: the frozen cross matrix of " +
                                            std::string(sd == 0 ? "test" : "trial") + " node " +
                                            std::to_string(st[1]) + " is singular at this wavenumber");
    }
    if (st[0] == 2) throw Failure(NCA_ERR_CUDA, "internal: a frozen cross block exceeds its planned capacity");
    launch_transpose_blocks<double2>(Xout, d.xoff.p, d.nrows.p, d.rank.p, d.xoff.p, d.nnodes, XTout, s);
    CK(cudaGetLastError());
}

// Near-field stores: one block per near pair (test CSR order) and its transpose (trial CSR
// order), with the pair lists and transposition plans kept for refills. Returns the entries.
int64_t build_near(nca_core *c, cudaStream_t s, std::vector<int64_t> *ntoff_out = nullptr) {
    const nca::Partition &P = c->part;
    const nca::Tree &Tt = c->tree[0], &Ts = c->tree[1];
    const int64_t nnear = P.nearnodes.size();
    c->h_noff.assign(Tt.nnodes + 1, 0);
    c->h_ncols.assign(Tt.nnodes, 0);
    c->h_nfoff.assign(nnear + 1, 0);
    std::vector<int32_t> near_t(nnear);
    int64_t near_entries = 0;
    for (int t = 0; t < Tt.nnodes; ++t) {
        int col = 0;
        for (int i = P.nearptr[t]; i < P.nearptr[t + 1]; ++i) {
            near_t[i] = t;
            const int ms = Ts.size(P.nearnodes[i]);
            col += ms;
            const int64_t e = int64_t(Tt.size(t)) * ms;
            near_entries += e;
            c->h_nfoff[i + 1] = c->h_nfoff[i] + pad2(e);
        }
        c->h_ncols[t] = col;
        c->h_noff[t + 1] = c->h_noff[t] + int64_t(Tt.size(t)) * col;
    }
    const int64_t ntn = P.tnearnodes.size();
    std::vector<int32_t> ntr_rows(ntn), ntr_cols(ntn);
    std::vector<int64_t> ntr_in(ntn), h_ntoff(ntn + 1, 0);
    for (int sn = 0; sn < Ts.nnodes; ++sn)
        for (int k = P.tnearptr[sn]; k < P.tnearptr[sn + 1]; ++k) {
            const int t = P.tnearnodes[k];
            auto it = std::lower_bound(P.nearnodes.begin() + P.nearptr[t], P.nearnodes.begin() + P.nearptr[t + 1], sn);
            ntr_in[k] = c->h_nfoff[it - P.nearnodes.begin()];
            ntr_rows[k] = Tt.size(t);
            ntr_cols[k] = Ts.size(sn);
            h_ntoff[k + 1] = h_ntoff[k] + pad2(int64_t(Tt.size(t)) * Ts.size(sn));
        }
    c->nearptr.upload(P.nearptr, s);
    c->nearnodes.upload(P.nearnodes, s);
    c->tnearptr.upload(P.tnearptr, s);
    c->tnearnodes.upload(P.tnearnodes, s);
    c->nfoff.upload(c->h_nfoff, s);
    c->ntoff.upload(h_ntoff, s);
    c->N.alloc(size_t(c->h_nfoff.back()));
    c->NT.alloc(size_t(h_ntoff.back()));
    c->near_t.upload(near_t, s);
    c->ntr_in.upload(ntr_in, s);
    c->ntr_rows.upload(ntr_rows, s);
    c->ntr_cols.upload(ntr_cols, s);
    c->n_ntr = ntn;
    fill_near(c, c->K, c->N.p, c->NT.p, s);
    if (ntoff_out) *ntoff_out = std::move(h_ntoff);
    return near_entries;
}

// Raises k_level_compress's dynamic shared-memory limit on the current device to at least sm and
// never lowers it, so that a build on another host thread keeps the limit its launches rely on.
void level_smem_at_least(size_t sm) {
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    cudaFuncAttributes fa{};
    CK(cudaFuncGetAttributes(&fa, k_level_compress));
    if (sm > size_t(fa.maxDynamicSharedSizeBytes)) {
        CK(cudaFuncSetAttribute(k_level_compress, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
        // all of the SM's unified L1/shared memory as shared: the CTAs per SM are bounded by it
        CK(cudaFuncSetAttribute(k_level_compress, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    }
}

// The skeleton of a built core as nca_core_save writes it: per side (node or item) the ranks, block
// rows, row pivots tau and column pivots sigma (maxrank per node), the interpolation operators X
// at their padded offsets and, for directional cores, the directional plan. Everything else
// (couplings, near field, product plans) is a function of the skeleton and is rebuilt by the
// build functions when they are given one.
struct SavedSide {
    std::vector<int32_t> rank, nrows, piv, cpiv, fpptr, fpidx;
    std::vector<int64_t> xoff;
    std::vector<double2> X;
    nca::DirSide plan;
};
struct SavedCore {
    SavedSide side[2];
};

void build_core(nca_core *c, const double *tp, int64_t nt, const double *sp, int64_t ns,
                const nca_build_opts *o, const SavedCore *sv = nullptr) {
    const int maxrank = c->maxrank;
    auto h0 = std::chrono::steady_clock::now();
    cudaStream_t s;
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{s};
    upload_tree(c->side[0], c->tree[0], tp, s);
    upload_tree(c->side[1], c->tree[1], sp, s);
    const nca::Partition &P = c->part;
    const bool iaca = o->compressor == NCA_COMPRESSOR_BOTTOMUP_IACA;
    // BottomUp(IACA): the nodes' far fields, centroids and the far trees' centres for the fused
    // kernel, which picks its geometric columns itself
    DBuf<int64_t> iffptr[2];
    DBuf<int32_t> iffnodes[2];
    DBuf<double> icent[2], icenter[2];
    // phase 1 on the device (tree mimicry); far field = own far nodes + ancestors'
    for (int sd = 0; sd < 2 && !sv; ++sd) {
        const nca::Tree &T = c->tree[sd];
        const std::vector<int32_t> &ptr = sd == 0 ? P.farptr : P.tfarptr;
        const std::vector<int32_t> &nodes = sd == 0 ? P.farnodes : P.tfarnodes;
        std::vector<int64_t> ffptr;
        std::vector<int32_t> ffnodes;
        parallel_csr(
            T.nnodes,
            [&](int t, std::vector<int32_t> &ff) {
                ff.clear();
                for (int a = t; a >= 0; a = T.parent[a])
                    ff.insert(ff.end(), nodes.begin() + ptr[a], nodes.begin() + ptr[a + 1]);
            },
            ffptr, ffnodes);
        if (iaca) {
            // the far points a node can offer, capped at maxrank, size its X slot (plan_side)
            const nca::Tree &Ft = c->tree[1 - sd];
            std::vector<int32_t> &fp = c->side[sd].h_fpptr;
            fp.assign(T.nnodes + 1, 0);
            for (int t = 0; t < T.nnodes; ++t) {
                int64_t n = 0;
                for (int64_t q = ffptr[t]; q < ffptr[t + 1] && n < maxrank; ++q) n += Ft.size(ffnodes[q]);
                fp[t + 1] = fp[t] + int32_t(std::min<int64_t>(n, maxrank));
            }
            iffptr[sd].upload(ffptr, s);
            iffnodes[sd].upload(ffnodes, s);
            icent[sd].upload(cluster_centroids(T, sd == 0 ? tp : sp), s);
            icenter[sd].upload(Ft.center, s);
            continue;
        }
        device_farpivots(T, sd == 0 ? tp : sp, c->tree[1 - sd], c->side[1 - sd], T.nnodes, ffptr, ffnodes, nullptr,
                         maxrank, s, c->side[sd].h_fpptr, c->side[sd].fpptr, c->side[sd].fpidx,
                         &c->side[sd].h_fpidx);
    }
    auto h1 = std::chrono::steady_clock::now();
    cudaEvent_t ev0, ev1;
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } eg{ev0, ev1};
    DBuf<int32_t> status;
    status.alloc(4);  // [flag, node, a, b]
    CK(cudaEventRecord(ev0, s));
    for (int sd = 0; sd < 2; ++sd) {
        DevSide &d = c->side[sd];
        const nca::Tree &T = c->tree[sd];
        if (sv) {
            // a saved skeleton: the operators and pivots as the build left them
            const SavedSide &v = sv->side[sd];
            d.h_xoff = v.xoff;
            d.xoff.upload(d.h_xoff, s);
            d.X.upload(v.X, s);
            d.rank.upload(v.rank, s);
            d.nrows.upload(v.nrows, s);
            d.piv.upload(v.piv, s);
            d.cpiv.upload(v.cpiv, s);
            d.h_rank = v.rank;
            d.h_nrows = v.nrows;
            d.h_piv = v.piv;
            d.h_fpptr = v.fpptr;
            d.h_fpidx = v.fpidx;
            plan_apply(d, T, s);
            d.XT.alloc(d.X.n);
            launch_transpose_blocks<double2>(d.X.p, d.xoff.p, d.nrows.p, d.rank.p, d.xoff.p, T.nnodes, d.XT.p, s);
            CK(cudaGetLastError());
            continue;
        }
        std::vector<int32_t> lv_ptr, lv_nodes;
        std::vector<int> lv_mcap, lv_ncap;
        plan_side(d, T, maxrank, lv_ptr, lv_nodes, lv_mcap, lv_ncap);
        d.xoff.upload(d.h_xoff, s);
        d.X.alloc(size_t(d.h_xoff.back()));
        d.rank.alloc(T.nnodes);
        d.rank.zero(s);
        d.nrows.alloc(T.nnodes);
        d.nrows.zero(s);
        d.piv.alloc(size_t(T.nnodes) * maxrank);
        d.cpiv.alloc(size_t(T.nnodes) * maxrank);
        DBuf<int32_t> nodes;
        nodes.upload(lv_nodes, s);
        status.zero(s);
        LevelArgs a{};
        a.K = c->K;
        a.side = sd;
        a.own_pts = d.pts.p;
        a.far_pts = c->side[1 - sd].pts.p;
        a.perm = d.perm.p;
        a.begin = d.begin.p;
        a.end = d.end.p;
        a.firstchild = d.firstchild.p;
        a.nchildren = d.nchildren.p;
        a.fpptr = d.fpptr.p;
        a.fpidx = d.fpidx.p;
        a.rank = d.rank.p;
        a.nrows = d.nrows.p;
        a.piv = d.piv.p;
        a.cpiv = d.cpiv.p;
        a.X = d.X.p;
        a.xoff = d.xoff.p;
        a.maxrank = maxrank;
        a.tol = sd == 0 ? o->tol_test : o->tol_trial;
        a.sampled = o->sampled;
        a.status = status.p;
        if (iaca) {
            const DevSide &fs = c->side[1 - sd];
            IacaArgs ia{};
            ia.mim.begin = fs.begin.p;
            ia.mim.end = fs.end.p;
            ia.mim.firstchild = fs.firstchild.p;
            ia.mim.nchildren = fs.nchildren.p;
            ia.mim.perm = fs.perm.p;
            ia.mim.center = icenter[sd].p;
            ia.mim.pts = fs.pts.p;
            ia.mim.nitems = T.nnodes;
            ia.mim.ffptr = iffptr[sd].p;
            ia.mim.ffnodes = iffnodes[sd].p;
            ia.mim.item_node = nullptr;
            ia.mim.centroid = icent[sd].p;
            ia.mim.maxrank = maxrank;
            ia.K = c->K;
            ia.side = sd;
            ia.own_pts = d.pts.p;
            ia.perm = d.perm.p;
            ia.begin = d.begin.p;
            ia.end = d.end.p;
            ia.firstchild = d.firstchild.p;
            ia.nchildren = d.nchildren.p;
            ia.rank = d.rank.p;
            ia.nrows = d.nrows.p;
            ia.piv = d.piv.p;
            ia.cpiv = d.cpiv.p;
            ia.X = d.X.p;
            ia.xoff = d.xoff.p;
            ia.maxrank = maxrank;
            ia.tol = a.tol;
            ia.status = status.p;
            for (size_t l = 0; l + 1 < lv_ptr.size(); ++l) {
                const int cnt = lv_ptr[l + 1] - lv_ptr[l];
                if (cnt == 0) continue;
                if (lv_mcap[l] > nca::iaca_max_rows())
                    throw Failure(NCA_ERR_ARG, "a cluster block has up to " + std::to_string(lv_mcap[l]) +
                                                   " rows; the IACA kernel holds at most " +
                                                   std::to_string(nca::iaca_max_rows()) + " (reduce the leaf size)");
                ia.items = nodes.p + lv_ptr[l];
                ia.nitems = cnt;
                launch_iaca(ia, lv_mcap[l], s);
                CK(cudaGetLastError());
            }
        } else {
            size_t maxsm = 0;
            for (size_t l = 0; l + 1 < lv_ptr.size(); ++l)
                maxsm = std::max(maxsm, level_smem_bytes(lv_mcap[l], lv_ncap[l]));
            if (maxsm > size_t(kMaxSmem))
                throw Failure(NCA_ERR_ARG,
                              "a level block does not fit in shared memory (reduce the leaf size or maxrank)");
            level_smem_at_least(maxsm);
            for (size_t l = 0; l + 1 < lv_ptr.size(); ++l) {
                int cnt = lv_ptr[l + 1] - lv_ptr[l];
                if (cnt == 0) continue;
                size_t sm = level_smem_bytes(lv_mcap[l], lv_ncap[l]);
                k_level_compress<<<cnt, 256, sm, s>>>(a, nodes.p + lv_ptr[l], lv_mcap[l], lv_ncap[l]);
                CK(cudaGetLastError());
            }
        }
        std::vector<int32_t> st = status.download(s);
        if (st[0] == 1) {
            set_singular(sd, st[1], st[2], st[3]);
            throw Failure(NCA_ERR_SINGULAR,
                          "SingularCrossMatrixError: the cross matrix of " + std::string(sd == 0 ? "test" : "trial") +
                              " node " + std::to_string(st[1]) + " is singular - " + std::to_string(st[2]) +
                              " pivots were selected but only " + std::to_string(st[3]) +
                              " of them are linearly independent (coincident points?)");
        }
        if (st[0] == 2) throw Failure(NCA_ERR_ARG, "internal: level block exceeds its planned capacity");
        if (st[0] == 3) throw Failure(NCA_ERR_CUDA, "internal: tree mimicry ran out of far points");
        d.h_rank = d.rank.download(s);
        d.h_nrows = d.nrows.download(s);
        d.h_piv = d.piv.download(s);
        if (iaca) {
            // the far pivots of a BottomUp(IACA) core are its column pivots sigma
            const std::vector<int32_t> cp = d.cpiv.download(s);
            d.h_fpptr.assign(T.nnodes + 1, 0);
            d.h_fpidx.clear();
            for (int t = 0; t < T.nnodes; ++t) {
                d.h_fpidx.insert(d.h_fpidx.end(), cp.begin() + int64_t(t) * maxrank,
                                 cp.begin() + int64_t(t) * maxrank + d.h_rank[t]);
                d.h_fpptr[t + 1] = int32_t(d.h_fpidx.size());
            }
        }
        plan_apply(d, T, s);
        d.XT.alloc(d.X.n);
        launch_transpose_blocks<double2>(d.X.p, d.xoff.p, d.nrows.p, d.rank.p, d.xoff.p, T.nnodes, d.XT.p, s);
        CK(cudaGetLastError());
    }
    // couplings S_ts = K[tau_t, sigma_s] in test CSR order, and their transposes in trial CSR order
    const nca::Tree &Tt = c->tree[0], &Ts = c->tree[1];
    const std::vector<int32_t> &rk_t = c->side[0].h_rank, &rk_s = c->side[1].h_rank;
    const int64_t npairs = P.farnodes.size();
    std::vector<int32_t> pair_t(npairs), pair_s(P.farnodes.begin(), P.farnodes.end());
    c->h_cfoff.assign(npairs + 1, 0);
    int64_t coupling_entries = 0;
    for (int t = 0; t < Tt.nnodes; ++t)
        for (int i = P.farptr[t]; i < P.farptr[t + 1]; ++i) {
            pair_t[i] = t;
            const int64_t e = int64_t(rk_t[t]) * rk_s[P.farnodes[i]];
            coupling_entries += e;
            c->h_cfoff[i + 1] = c->h_cfoff[i] + pad2(e);
        }
    c->farptr.upload(P.farptr, s);
    c->farnodes.upload(P.farnodes, s);
    c->tfarptr.upload(P.tfarptr, s);
    c->tfarnodes.upload(P.tfarnodes, s);
    const int64_t ntf = P.tfarnodes.size();
    std::vector<int32_t> tfarpair(ntf), tr_rows(ntf), tr_cols(ntf);
    std::vector<int64_t> tr_in(ntf), h_ctoff(ntf + 1, 0);
    for (int sn = 0; sn < Ts.nnodes; ++sn)
        for (int k = P.tfarptr[sn]; k < P.tfarptr[sn + 1]; ++k) {
            const int t = P.tfarnodes[k];
            auto it = std::lower_bound(P.farnodes.begin() + P.farptr[t], P.farnodes.begin() + P.farptr[t + 1], sn);
            const int pair = int(it - P.farnodes.begin());
            tfarpair[k] = pair;
            tr_in[k] = c->h_cfoff[pair];
            tr_rows[k] = rk_t[t];
            tr_cols[k] = rk_s[sn];
            h_ctoff[k + 1] = h_ctoff[k] + pad2(int64_t(rk_t[t]) * rk_s[sn]);
        }
    c->tfarpair.upload(tfarpair, s);
    c->cfoff.upload(c->h_cfoff, s);
    c->ctoff.upload(h_ctoff, s);
    c->C.alloc(size_t(c->h_cfoff.back()));
    c->CT.alloc(size_t(h_ctoff.back()));
    c->cpair_t.upload(pair_t, s);
    c->ctr_in.upload(tr_in, s);
    c->ctr_rows.upload(tr_rows, s);
    c->ctr_cols.upload(tr_cols, s);
    c->n_ctr = ntf;
    fill_couplings(c, c->K, c->C.p, c->CT.p, s);
    CK(cudaStreamSynchronize(s));
    // output nodes of the coupling stage, largest work first (shorter tail of the last wave)
    std::vector<int32_t> fwd, rev;
    std::vector<int64_t> wf(Tt.nnodes, 0), wr(Ts.nnodes, 0);
    for (int t = 0; t < Tt.nnodes; ++t) {
        if (rk_t[t] <= 0) continue;
        fwd.push_back(t);
        for (int i = P.farptr[t]; i < P.farptr[t + 1]; ++i) wf[t] += int64_t(rk_t[t]) * rk_s[P.farnodes[i]];
    }
    for (int sn = 0; sn < Ts.nnodes; ++sn) {
        if (rk_s[sn] <= 0) continue;
        rev.push_back(sn);
        for (int k = P.tfarptr[sn]; k < P.tfarptr[sn + 1]; ++k) wr[sn] += int64_t(rk_s[sn]) * rk_t[P.tfarnodes[k]];
    }
    std::stable_sort(fwd.begin(), fwd.end(), [&](int a, int b) { return wf[a] > wf[b]; });
    std::stable_sort(rev.begin(), rev.end(), [&](int a, int b) { return wr[a] > wr[b]; });
    c->n_couple_fwd = int(fwd.size());
    c->n_couple_rev = int(rev.size());
    c->couple_fwd.upload(fwd, s);
    c->couple_rev.upload(rev, s);
    // leaves of both sides, largest work (near columns + own basis) first
    for (int sd = 0; sd < 2; ++sd) {
        const nca::Tree &T = c->tree[sd];
        const std::vector<int32_t> &ptr = sd == 0 ? P.nearptr : P.tnearptr;
        const std::vector<int32_t> &nodes = sd == 0 ? P.nearnodes : P.tnearnodes;
        const nca::Tree &F = c->tree[1 - sd];
        std::vector<int64_t> work(T.nnodes, 0);
        std::vector<int32_t> leaves;
        for (int t = 0; t < T.nnodes; ++t) {
            if (!T.isleaf(t)) continue;
            leaves.push_back(t);
            work[t] = c->side[sd].h_rank[t];
            for (int i = ptr[t]; i < ptr[t + 1]; ++i) work[t] += F.size(nodes[i]);
            work[t] *= T.size(t);
        }
        std::stable_sort(leaves.begin(), leaves.end(), [&](int a, int b) { return work[a] > work[b]; });
        c->side[sd].leaves.upload(leaves, s);
    }
    const int64_t near_entries = build_near(c, s);
    if (c->f32) make_f32_copies(c, s);
    CK(cudaEventRecord(ev1, s));
    CK(cudaStreamSynchronize(s));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ev0, ev1));
    auto h2 = std::chrono::steady_clock::now();
    nca_core_info &I = c->info;
    I.ntest = nt;
    I.ntrial = ns;
    I.nnodes_test = Tt.nnodes;
    I.nnodes_trial = Ts.nnodes;
    I.ncoeff_test = c->side[0].h_cptr.back();
    I.ncoeff_trial = c->side[1].h_cptr.back();
    I.near_entries = near_entries;
    I.coupling_entries = coupling_entries;
    for (int sd = 0; sd < 2; ++sd) {
        int64_t basis = 0, transfer = 0;
        const nca::Tree &T = c->tree[sd];
        for (int node = 0; node < T.nnodes; ++node) {
            int64_t e = int64_t(c->side[sd].h_nrows[node]) * c->side[sd].h_rank[node];
            (T.isleaf(node) ? basis : transfer) += e;
        }
        (sd == 0 ? I.basis_entries_test : I.basis_entries_trial) = basis;
        (sd == 0 ? I.transfer_entries_test : I.transfer_entries_trial) = transfer;
    }
    I.nfarpairs = npairs;
    I.nnearpairs = int64_t(P.nearnodes.size());
    I.build_seconds = ms * 1e-3;
    I.build_seconds_host = std::chrono::duration<double>(h1 - h0).count() +
                           std::chrono::duration<double>(h2 - h1).count() - ms * 1e-3;
}

// ---- directional (wideband) build ------------------------------------------------------
// Bases are built per item (cluster, direction) by BottomUp(IACA) (k_iaca, one warp per item, level
// by level): the rows of a basis item are its cluster's points, those of a nested item the pivots
// of its children's items in the mapped directions; the geometric columns come from tree mimicry
// over the item's directional far field. The product stages then become block-sparse gathers over one vector arena, each
// block stored contiguously: up (item <- its children's items or its cluster's x slice), coupling
// (item <- far items), down (child item <- its parents' items: several parent directions can map
// onto one child direction, so the children gather), leaves (leaf <- every basis item whose
// cluster contains it, and the near blocks).

// complex-FP32 products of at least this many right-hand sides run their gathers on the tensor
// cores (NCA_TC_COLUMNS overrides it; a large value keeps them on the FP32 pipe)
const int kTensorCoreColumns = [] {
    const char *v = std::getenv("NCA_TC_COLUMNS");
    return v ? std::max(1, std::atoi(v)) : 32;
}();
// launch groups of small outputs (mean block entries per output below this) run on the gather
// kernels that keep a warp per output
constexpr double kSmallGroupWork = 8192.0;
// a launch group the all-column FP32 kernel takes (complex-FP32 products of two or more columns)
bool wide_group(int maxrows, double work) { return work < kSmallGroupWork && gather_wide_fits(maxrows); }

struct StageBuilder {
    std::vector<int32_t> group_ptr{0};
    std::vector<int> group_maxrows;
    std::vector<double> group_work;
    hvec<int32_t> rows, segptr{0}, w;
    hvec<int64_t> out, moff, voff, work;
    // sub-matrix copies from the source store into the stage store
    hvec<int64_t> soff, doff;
    hvec<int32_t> sld, crows, ccols;
    int64_t store = 0;
    int cur_max = 0;
    // room for the outputs, segments and copies a stage is known to have at most
    void reserve(size_t outputs, size_t segments, size_t copies) {
        rows.reserve(outputs);
        out.reserve(outputs);
        work.reserve(outputs);
        segptr.reserve(outputs + 1);
        moff.reserve(segments);
        w.reserve(segments);
        voff.reserve(segments);
        soff.reserve(copies);
        doff.reserve(copies);
        sld.reserve(copies);
        crows.reserve(copies);
        ccols.reserve(copies);
    }
    void begin_output(int32_t R, int64_t o) {
        rows.push_back(R);
        out.push_back(o);
        work.push_back(0);
        cur_max = std::max(cur_max, R);
    }
    void segment(int64_t mo, int32_t width, int64_t vo) {
        moff.push_back(mo);
        w.push_back(width);
        voff.push_back(vo);
        work.back() += int64_t(rows.back()) * width;
    }
    // a block copied from the source store (R x C at offset so, leading dimension ld) into the
    // stage store; returns its offset there
    int64_t copy(int64_t so, int32_t ld, int32_t R, int32_t C) {
        const int64_t d = store;
        soff.push_back(so);
        sld.push_back(ld);
        crows.push_back(R);
        ccols.push_back(C);
        doff.push_back(d);
        store += pad2(int64_t(R) * C);
        return d;
    }
    void end_output() { segptr.push_back(int32_t(moff.size())); }
    void end_group() {
        const int32_t b = group_ptr.back(), e = int32_t(rows.size());
        double sum = 0.0;
        for (int32_t i = b; i < e; ++i) sum += double(work[i]);
        group_work.push_back(e > b ? sum / double(e - b) : 0.0);
        group_ptr.push_back(e);
        group_maxrows.push_back(std::max(cur_max, 1));
        cur_max = 0;
    }
    // one line per launch group on stderr: outputs, largest and mean output rows, segments and
    // vector rows per output, block entries
    void print_stats(const char *tag) const {
        for (size_t g = 0; g + 1 < group_ptr.size(); ++g) {
            const int32_t b = group_ptr[g], e = group_ptr[g + 1];
            int64_t R = 0, nseg = 0, vrows = 0, ent = 0;
            for (int32_t i = b; i < e; ++i) {
                R += rows[i];
                nseg += segptr[i + 1] - segptr[i];
                for (int32_t k = segptr[i]; k < segptr[i + 1]; ++k) vrows += w[k];
                ent += work[i];
            }
            const double n = double(std::max(e - b, 1));
            fprintf(stderr,
                    "nca stats %-10s group %2zu: %8d outputs, rows max %3d mean %6.2f, segments %6.2f, "
                    "vector rows %8.2f, entries %12lld, work %8.1f\n",
                    tag, g, e - b, group_maxrows[g], double(R) / n, double(nseg) / n, double(vrows) / n,
                    (long long)ent, group_work[g]);
        }
    }
    // adds dy to the vector rows of the segments that read the store (not the second store's near
    // blocks) and, with outs, to the outputs' rows: a plan listed before the arena offset was known
    void shift(int64_t dy, bool outs) {
        for (size_t k = 0; k < moff.size(); ++k)
            if (moff[k] >= 0) voff[k] += dy;
        if (outs)
            for (int64_t &o : out) o += dy;
    }
    // uploads the plan; with a source, allocates the stage store and copies its blocks
    void finish(GatherStage &G, const double2 *src, cudaStream_t s, const char *tag = nullptr,
                const std::function<void(const std::string &)> &mark = {}) {
        if (tag && getenv("NCA_DIR_STATS")) print_stats(tag);
        // outputs of each group largest work first (shorter tail of the last wave): a stable
        // counting sort on the work, linear in the outputs
        hvec<int32_t> order(rows.size());
        std::vector<int64_t> cnt;
        for (size_t g = 0; g + 1 < group_ptr.size(); ++g) {
            const int32_t b = group_ptr[g], e = group_ptr[g + 1];
            if (e <= b) continue;
            int64_t wmax = 0;
            for (int32_t i = b; i < e; ++i) wmax = std::max(wmax, work[i]);
            if (wmax > 8 * int64_t(e - b) + 4096) {
                // few outputs of large work (the leaves): a comparison sort, same order
                for (int32_t i = b; i < e; ++i) order[i] = i;
                std::stable_sort(order.begin() + b, order.begin() + e,
                                 [&](int32_t x, int32_t y) { return work[x] > work[y]; });
                continue;
            }
            cnt.assign(size_t(wmax) + 2, 0);
            for (int32_t i = b; i < e; ++i) ++cnt[size_t(wmax - work[i]) + 1];
            for (size_t k = 1; k < cnt.size(); ++k) cnt[k] += cnt[k - 1];
            for (int32_t i = b; i < e; ++i) order[size_t(b + cnt[size_t(wmax - work[i])]++)] = i;
        }
        // fn(k, i0, i1) over nparts consecutive ranges of [b, e), on threads of their own when
        // the range is long
        auto in_parts = [](int32_t b, int32_t e, int nparts, auto fn) {
            if (nparts <= 1) {
                fn(0, b, e);
                return;
            }
            std::vector<std::thread> pool;
            for (int k = 1; k < nparts; ++k)
                pool.emplace_back([&, k] {
                    fn(k, int32_t(b + int64_t(e - b) * k / nparts), int32_t(b + int64_t(e - b) * (k + 1) / nparts));
                });
            fn(0, b, int32_t(b + int64_t(e - b) / nparts));
            for (auto &th : pool) th.join();
        };
        auto parts_of = [](int32_t n) { return std::max(1, std::min(8, int(n / 65536))); };
        // Records of the all-column FP32 kernel (groups of small outputs): inside a group the
        // records of one row class (the kernel's register tile) are contiguous, largest work
        // first inside a class: one launch per class
        // the vector rows an output reads: its work over its rows (work = rows x widths, summed
        // while listing), so the segments need not be visited again
        auto width = [&](int32_t o) -> int32_t {
            if (rows[o] > 0) return int32_t(work[o] / rows[o]);
            int32_t W = 0;
            for (int32_t k = segptr[o]; k < segptr[o + 1]; ++k) W += w[k];
            return W;
        };
        G.wide_gptr.assign(1, 0);
        G.wide_begin.clear();
        G.wide_count.clear();
        G.wide_nr.clear();
        hvec<WideOut> rec;
        rec.reserve(order.size());
        for (size_t g = 0; g + 1 < group_ptr.size(); ++g) {
            const int32_t b = group_ptr[g], e = group_ptr[g + 1];
            if (e > b && wide_group(group_maxrows[g], group_work[g])) {
                // each part counts its classes; a part's records of a class follow those of the
                // parts before it, so the records are those of one pass in order
                const int np = parts_of(e - b);
                std::vector<int32_t> pc(size_t(np) * 34, 0);  // [part][class]
                in_parts(b, e, np, [&](int k, int32_t i0, int32_t i1) {
                    int32_t *cc = pc.data() + size_t(k) * 34;
                    for (int32_t i = i0; i < i1; ++i) ++cc[wide_rows_class(rows[order[i]])];
                });
                int32_t at = int32_t(rec.size());
                for (int c = 0; c < 34; ++c) {
                    int32_t n = 0;
                    for (int k = 0; k < np; ++k) {
                        const int32_t q = pc[size_t(k) * 34 + c];
                        pc[size_t(k) * 34 + c] = at + n;  // the part's first slot of the class
                        n += q;
                    }
                    if (n) {
                        G.wide_begin.push_back(at);
                        G.wide_count.push_back(n);
                        G.wide_nr.push_back(c);
                    }
                    at += n;
                }
                rec.resize(size_t(at));
                in_parts(b, e, np, [&](int k, int32_t i0, int32_t i1) {
                    int32_t *slot = pc.data() + size_t(k) * 34;
                    for (int32_t i = i0; i < i1; ++i) {
                        const int32_t o = order[i];
                        rec[size_t(slot[wide_rows_class(rows[o])]++)] =
                            WideOut{rows[o], width(o), segptr[o], segptr[o + 1], out[o], rows[o], 0};
                    }
                });
            }
            G.wide_gptr.push_back(int32_t(G.wide_begin.size()));
        }
        G.group_ptr = group_ptr;
        G.group_maxrows = group_maxrows;
        G.group_work = group_work;
        // records of the tensor-core gathers: the groups the all-column FP32 kernel does not take
        // (left zero elsewhere)
        // (only if some group takes them)
        bool any_tc = false;
        for (size_t g = 0; g + 1 < group_ptr.size(); ++g) any_tc = any_tc || !wide_group(group_maxrows[g], group_work[g]);
        hvec<WideOut> trec(any_tc ? order.size() : 0);
        for (size_t g = 0; any_tc && g + 1 < group_ptr.size(); ++g) {
            if (wide_group(group_maxrows[g], group_work[g])) continue;
            const int32_t b = group_ptr[g], e = group_ptr[g + 1];
            in_parts(b, e, parts_of(e - b), [&](int, int32_t i0, int32_t i1) {
                for (int32_t i = i0; i < i1; ++i) {
                    const int32_t o = order[i];
                    trec[i] = WideOut{rows[o], width(o), segptr[o], segptr[o + 1], out[o], rows[o], 0};
                }
            });
        }
        if (mark)
            mark("records (" + std::to_string(rows.size()) + " outputs, " + std::to_string(w.size()) + " segments, " +
                 std::to_string(crows.size()) + " copies)");
        const size_t bytes = sizeof(int32_t) * (order.size() + rows.size() + segptr.size() + w.size() + sld.size() +
                                                crows.size() + ccols.size()) +
                             sizeof(WideOut) * (rec.size() + trec.size()) +
                             sizeof(int64_t) * (out.size() + moff.size() + voff.size() + soff.size() + doff.size()) +
                             16 * 16;
        StagedUploads up(bytes, s);
        up.up(G.outputs, order);
        up.up(G.wout, rec);
        up.up(G.tout, trec);
        up.up(G.rows, rows);
        up.up(G.out, out);
        up.up(G.segptr, segptr);
        up.up(G.moff, moff);
        up.up(G.w, w);
        up.up(G.voff, voff);
        if (src && !crows.empty()) {
            up.up(G.c_soff, soff);
            up.up(G.c_doff, doff);
            up.up(G.c_ld, sld);
            up.up(G.c_rows, crows);
            up.up(G.c_cols, ccols);
        }
        up.flush();
        if (mark) mark("plan uploaded (" + std::to_string(bytes >> 20) + " MiB)");
        if (!src) return;
        G.M.alloc(size_t(store));
        if (mark) mark("store allocated");
        G.entries = 0;
        for (size_t i = 0; i < crows.size(); ++i) G.entries += int64_t(crows[i]) * ccols[i];
        G.ncopies = int64_t(crows.size());
        if (!crows.empty()) {
            launch_copy_blocks<double2>(src, G.c_soff.p, G.c_ld.p, G.c_rows.p, G.c_cols.p, G.c_doff.p, G.ncopies,
                                        G.M.p, s);
            CK(cudaGetLastError());
            CK(cudaStreamSynchronize(s));
        }
    }
};

// fn(0) .. fn(n - 1) on n host threads (the caller and n - 1 more, all on the core's device); the
// first failure in task order, with its singular-matrix record, is rethrown on the caller once
// all are done
template <typename F>
void on_threads(int device, int n, F fn) {
    std::vector<std::exception_ptr> err(n);
    std::vector<std::array<int, 4>> sing(n);
    auto run = [&](int i) {
        try {
            if (i) CK(cudaSetDevice(device));
            fn(i);
        } catch (...) {
            err[i] = std::current_exception();
            std::copy(g_singular, g_singular + 4, sing[i].begin());
        }
    };
    std::vector<std::thread> pool;
    for (int i = 1; i < n; ++i) {
        try {
            pool.emplace_back(run, i);
        } catch (const std::system_error &) {
            run(i);  // no thread to be had: the task runs here, in order
        }
    }
    run(0);
    for (auto &th : pool) th.join();
    for (int i = 0; i < n; ++i)
        if (err[i]) {
            set_singular(sing[i][0], sing[i][1], sing[i][2], sing[i][3]);
            std::rethrow_exception(err[i]);
        }
}

// Wall-clock marks of the build's phases; with NCA_BUILD_TIMING set they are printed to stderr
// when the build ends (the reference prints its batched compressor's phases under
// NCA_BATCHED_TIMING, src/compressors/batchedbottomup.jl:74-78).
struct PhaseTimer {
    bool on = std::getenv("NCA_BUILD_TIMING") != nullptr;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    std::mutex mu;
    std::vector<std::pair<double, std::string>> marks;
    void mark(const std::string &what) {
        if (!on) return;
        const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::lock_guard<std::mutex> g(mu);
        marks.emplace_back(t, what);
    }
    ~PhaseTimer() {
        if (!on) return;
        std::sort(marks.begin(), marks.end());
        for (const auto &m : marks) std::fprintf(stderr, "nca build %9.4f s  %s\n", m.first, m.second.c_str());
    }
};

// BottomUp(IACA) of one side of a directional core: the items' far fields, then one k_iaca launch
// per level (deepest first), each level's operators compacted to the ranks found; leaves the
// side's X, h_xoff, ranks and rows in d.
void compress_dir_side(nca_core *c, DirItems &d, int sd, const double *ownpts,
                       const std::vector<std::vector<int32_t>> &bylevel, cudaStream_t s, const nca_build_opts *o,
                       PhaseTimer &timer, const std::string &side, const std::function<void()> &ranks_known,
                       cudaStream_t hs) {
    const int maxrank = c->maxrank;
    const nca::DirSide &pl = d.plan;
    const nca::Tree &T = c->tree[sd], &Ft = c->tree[1 - sd];
    DevSide &ds = c->side[sd];
    const DevSide &fs = c->side[1 - sd];
    const int ni = d.nitems;
    // The items' directional far fields (dirfarfield, in the reference's order) and the far points
    // each can offer (capped at maxrank), listed one level at a time on the host threads: a level's
    // lists are made while the device compresses the level below it. An item without far nodes
    // is not compressed; its empty range leaves the level's CSR over the remaining items intact.
    struct LevelFar {
        std::vector<int32_t> items, farpts;  // the level's items with far points, and their counts
        hvec<int64_t> ptr;                    // CSR over those items (positional)
        hvec<int32_t> nodes;
    };
    auto list_level = [&, maxrank](int lev) {
        LevelFar L;
        const std::vector<int32_t> &cand = bylevel[lev];
        hvec<int64_t> ptr;
        parallel_csr(
            int(cand.size()), [&](int i, std::vector<int32_t> &ff) { nca::item_farfield(T, pl, cand[i], ff); }, ptr,
            L.nodes);
        L.ptr.push_back(0);
        for (size_t i = 0; i < cand.size(); ++i) {
            int64_t n = 0;
            for (int64_t q = ptr[i]; q < ptr[i + 1] && n < maxrank; ++q) n += Ft.size(L.nodes[q]);
            if (n == 0) continue;
            L.items.push_back(cand[i]);
            L.farpts.push_back(int32_t(std::min<int64_t>(n, maxrank)));
            L.ptr.push_back(ptr[i + 1]);
        }
        return L;
    };
    // two levels listed ahead: the deepest level is small, and the next one's list would
    // otherwise hold up its launch
    std::vector<std::future<LevelFar>> far_of(size_t(std::max(T.nlevels, 0)));
    for (int lev = T.nlevels - 1; lev >= 0 && lev >= T.nlevels - 2; --lev)
        far_of[size_t(lev)] = std::async(std::launch::async, list_level, lev);
    const std::vector<double> centroid = cluster_centroids(T, ownpts);
    DBuf<int64_t> dffptr;
    DBuf<int32_t> dffnodes;
    DBuf<double> dcent, dcenter;
    {
        // through one page-locked block (pageable copies are staged by the driver, a few GB/s)
        const size_t bytes = sizeof(double) * (centroid.size() + Ft.center.size()) +
                             sizeof(int32_t) * (pl.item_node.size() + pl.item_basis.size() + pl.item_chptr.size() +
                                                pl.item_chidx.size()) +
                             6 * 16;
        StagedUploads up(bytes, s);
        up.up(dcent, centroid);
        up.up(dcenter, Ft.center);
        up.up(d.item_node, pl.item_node);
        up.up(d.item_basis, pl.item_basis);
        up.up(d.item_chptr, pl.item_chptr);
        up.up(d.item_chidx, pl.item_chidx);
    }
    timer.mark(side + "centroids and items uploaded");
    // the side's items, level by level
    DBuf<int32_t> status;
    status.alloc(4);  // [flag, item, a, b]
    d.rank.alloc(std::max(ni, 1));
    d.rank.zero(s);
    d.nrows.alloc(std::max(ni, 1));
    d.nrows.zero(s);
    d.piv.alloc(size_t(std::max(ni, 1)) * maxrank);
    IacaArgs a{};
    a.mim.begin = fs.begin.p;
    a.mim.end = fs.end.p;
    a.mim.firstchild = fs.firstchild.p;
    a.mim.nchildren = fs.nchildren.p;
    a.mim.perm = fs.perm.p;
    a.mim.center = dcenter.p;
    a.mim.pts = fs.pts.p;
    a.mim.nitems = ni;
    a.mim.ffptr = dffptr.p;
    a.mim.ffnodes = dffnodes.p;
    a.mim.item_node = d.item_node.p;
    a.mim.centroid = dcent.p;
    a.mim.maxrank = maxrank;
    a.K = c->K;
    a.side = sd;
    a.own_pts = ds.pts.p;
    a.perm = ds.perm.p;
    a.begin = ds.begin.p;
    a.end = ds.end.p;
    a.firstchild = ds.firstchild.p;
    a.nchildren = ds.nchildren.p;
    a.item_basis = d.item_basis.p;
    a.item_chptr = d.item_chptr.p;
    a.item_chidx = d.item_chidx.p;
    a.rank = d.rank.p;
    a.nrows = d.nrows.p;
    a.piv = d.piv.p;
    d.cpiv.alloc(size_t(std::max(ni, 1)) * maxrank);
    a.cpiv = d.cpiv.p;
    timer.mark(side + "item arrays allocated");
    a.maxrank = maxrank;
    a.tol = sd == 0 ? o->tol_test : o->tol_trial;
    a.status = status.p;
    // Level by level, deepest first: the rows of a nested item are its children's actual
    // ranks, so each level's X is allocated for min(maxrank, rows, far points) columns, then
    // compacted to the ranks found before the next level runs.
    d.h_rank.assign(ni, 0);
    d.h_nrows.assign(ni, 0);
    std::vector<int64_t> cpos(ni, -1);
    std::vector<std::unique_ptr<DBuf<double2>>> levelX;
    std::vector<std::vector<int32_t>> levelItems;
    // scratch reused by every level (grown, never shrunk: no device-wide frees between levels);
    // the level's slot offsets, ranks and rows are indexed by position in the level's item list
    DBuf<int64_t> dlvoff, ddo;
    DBuf<int32_t> nodes, drk;
    DBuf<double2> chunk;
    // ranks and rows read back per level, through a block of the page-locked pool (returned
    // below, once the side's stream has synchronised)
    PinnedPool::Block hrank_block = PinnedPool::get().acquire(sizeof(int32_t) * 2 * size_t(std::max(ni, 1)));
    if (!hrank_block.p) throw Failure(NCA_ERR_CUDA, "no page-locked host memory for the rank read-back");
    struct BlockGuard {
        PinnedPool::Block b;
        cudaStream_t s;
        ~BlockGuard() {
            cudaStreamSynchronize(s);  // no read-back still lands in the block
            PinnedPool::get().release(b);
        }
    } hrank_guard{hrank_block, s};
    int32_t *const hrank = reinterpret_cast<int32_t *>(hrank_block.p);
    a.xoff_by_position = 1;
    int64_t total = 0;
    a.mim.ff_by_position = 1;
    for (int lev = T.nlevels - 1; lev >= 0; --lev) {
        const LevelFar far = far_of[size_t(lev)].get();
        timer.mark(side + "level " + std::to_string(lev) + " far field listed");
        if (lev >= 2) far_of[size_t(lev) - 2] = std::async(std::launch::async, list_level, lev - 2);
        const std::vector<int32_t> &items = far.items;
        std::vector<int64_t> lvoff;
        int mc = 0;
        int64_t bound = 0;
        for (size_t i = 0; i < items.size(); ++i) {
            const int it = items[i];
            int64_t m = 0;
            if (pl.item_basis[it]) {
                m = T.size(pl.item_node[it]);
            } else {
                for (int k = pl.item_chptr[it]; k < pl.item_chptr[it + 1]; ++k) m += d.h_rank[pl.item_chidx[k]];
            }
            const int64_t rb = std::min<int64_t>(std::min<int64_t>(maxrank, m), int64_t(far.farpts[i]));
            lvoff.push_back(bound);
            bound += pad2(m * rb);
            mc = int(std::max<int64_t>(mc, m));
        }
        if (items.empty()) continue;
        upload_reuse(dffptr, far.ptr, s, d.later);
        upload_reuse(dffnodes, far.nodes, s, d.later);
        a.mim.ffptr = dffptr.p;
        a.mim.ffnodes = dffnodes.p;
        if (mc > nca::iaca_max_rows())
            throw Failure(NCA_ERR_ARG, "a basis item has " + std::to_string(mc) +
                                           " rows; the IACA kernel holds at most " +
                                           std::to_string(nca::iaca_max_rows()) + " (reduce the leaf size)");
        if (!chunk.p || size_t(bound) > chunk.n) {
            chunk.defer(d.later);
            chunk.alloc_scratch(size_t(std::max<int64_t>(bound, 1)));
            timer.mark(side + "level " + std::to_string(lev) + " scratch of " + std::to_string(bound >> 16) +
                       " x 1 MiB allocated");
        }
        upload_reuse(dlvoff, lvoff, s, d.later);
        upload_reuse(nodes, items, s, d.later);
        const int nl = int(items.size());
        if (drk.n < 2 * size_t(nl)) {
            drk.defer(d.later);
            drk.alloc_scratch(2 * size_t(nl));
        }
        status.zero(s);
        a.X = chunk.p;
        a.xoff = dlvoff.p;
        a.items = nodes.p;
        a.nitems = nl;
        a.rank_pos = drk.p;
        launch_iaca(a, mc, s);
        CK(cudaGetLastError());
        const std::vector<int32_t> st = status.download(s);
        if (st[0] == 1) {
            set_singular(sd, st[1], st[2], st[3]);
            throw Failure(NCA_ERR_SINGULAR, "SingularCrossMatrixError: the cross matrix of " +
                                                std::string(sd == 0 ? "test" : "trial") + " item " +
                                                std::to_string(st[1]) + " is singular - " + std::to_string(st[2]) +
                                                " pivots were selected but only " + std::to_string(st[3]) +
                                                " of them are linearly independent");
        }
        if (st[0] == 2) throw Failure(NCA_ERR_ARG, "internal: an item exceeds the IACA kernel's row capacity");
        if (st[0] == 3) throw Failure(NCA_ERR_CUDA, "internal: tree mimicry ran out of far points");
        CK(cudaMemcpyAsync(hrank, drk.p, sizeof(int32_t) * 2 * nl, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        timer.mark(side + "level " + std::to_string(lev) + " IACA done");
        const int32_t *rk = hrank, *nr = hrank + nl;
        // compact this level: exact m x r blocks, back to back (one copy per item, rank-0 items
        // copy nothing; sources, rows and columns straight from the positional arrays)
        std::vector<int64_t> doff(nl);
        int64_t lt = 0;
        for (int i = 0; i < nl; ++i) {
            const int it = items[i];
            d.h_rank[it] = rk[i];
            d.h_nrows[it] = nr[i];
            cpos[it] = lt;
            doff[i] = lt;
            lt += pad2(int64_t(nr[i]) * rk[i]);
        }
        levelX.emplace_back(new DBuf<double2>());
        levelX.back()->alloc_scratch(size_t(std::max<int64_t>(lt, 1)));
        if (lt > 0) {
            // on the high-priority stream: its blocks start ahead of the other side's IACA blocks
            upload_reuse(ddo, doff, hs, d.later);
            launch_copy_blocks<double2>(chunk.p, dlvoff.p, drk.p + nl, drk.p + nl, drk.p, ddo.p, int64_t(nl),
                                        levelX.back()->p, hs);
            CK(cudaGetLastError());
            CK(cudaStreamSynchronize(hs));
        }
        levelItems.push_back(items);
        for (int it : items) cpos[it] += total;
        total += lt;
        timer.mark(side + "level " + std::to_string(lev) + " (" + std::to_string(items.size()) +
                   " items, up to " + std::to_string(mc) + " rows) compressed and compacted");
    }
    // one X for the side: the compacted levels back to back
    d.h_xoff.assign(ni + 1, 0);
    for (int it = 0; it < ni; ++it) d.h_xoff[it] = cpos[it] >= 0 ? cpos[it] : 0;
    d.h_xoff[ni] = total;
    ranks_known();  // the gather plans list from here while the levels are joined on the device
    d.X.alloc(size_t(std::max<int64_t>(total, 1)));
    {
        int64_t off = 0;
        for (size_t l = 0; l < levelX.size(); ++l) {
            int64_t lt = 0;
            for (int it : levelItems[l]) lt += pad2(int64_t(d.h_nrows[it]) * d.h_rank[it]);
            if (lt)
                CK(cudaMemcpyAsync(d.X.p + off, levelX[l]->p, sizeof(double2) * lt, cudaMemcpyDeviceToDevice,
                                   s));
            off += lt;
        }
        CK(cudaStreamSynchronize(s));
        for (auto &x : levelX) x->defer(d.later);
        levelX.clear();
    }
    for (auto *b : {&dffptr, &dlvoff, &ddo}) b->defer(d.later);
    for (auto *b : {&dffnodes, &status, &nodes, &drk}) b->defer(d.later);
    for (auto *b : {&dcent, &dcenter}) b->defer(d.later);
    chunk.defer(d.later);
}

void build_dir_core(nca_core *c, const double *tp, const double *sp, const nca_build_opts *o, const nca::Wideband &wb,
                    const SavedCore *sv = nullptr) {
    const int maxrank = c->maxrank;
    PhaseTimer timer;
    auto h0 = std::chrono::steady_clock::now();
    cudaStream_t s;
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{s};
    upload_tree(c->side[0], c->tree[0], tp, s);
    upload_tree(c->side[1], c->tree[1], sp, s);
    const nca::Partition &P = c->part;
    auto D = std::make_unique<DirCore>();
    const double *pts[2] = {tp, sp};
    // the two sides (and later the two orientations of the gather plans) are independent: each
    // runs on its own host thread and stream
    cudaStream_t s1;
    CK(cudaStreamCreateWithFlags(&s1, cudaStreamNonBlocking));
    StreamGuard sg1{s1};
    const cudaStream_t ss[2] = {s, s1};
    // high-priority streams for the short steps between a side's IACA levels (the compaction):
    // their blocks are scheduled before the pending blocks of the other side's IACA launch
    int prio_low = 0, prio_high = 0;
    CK(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    cudaStream_t h0s, h1s;
    CK(cudaStreamCreateWithPriority(&h0s, cudaStreamNonBlocking, prio_high));
    StreamGuard hg0{h0s};
    CK(cudaStreamCreateWithPriority(&h1s, cudaStreamNonBlocking, prio_high));
    StreamGuard hg1{h1s};
    const cudaStream_t hs[2] = {h0s, h1s};
    CK(cudaStreamSynchronize(s));
    cudaEvent_t ev0, ev1;
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } eg{ev0, ev1};
    CK(cudaEventRecord(ev0, s));
    // The near field depends on the trees and the partition only: it is built on a thread and
    // stream of its own while the sides plan their directions and compress (its offsets feed the
    // leaf plans).
    cudaStream_t s2;
    CK(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
    StreamGuard sg2{s2};
    std::vector<int64_t> h_ntoff;
    int64_t near_entries = 0;
    // complex-FP32 copy of a store, made on the stream that filled it (by the thread that did), so
    // that the copies overlap the rest of the build instead of following it
    auto to_f32 = [&](DBuf<double2> &src, DBuf<float2> &dst, cudaStream_t st) {
        if (!c->f32) return;
        dst.alloc(src.n);
        if (src.n) k_to_f32<<<launch_grid(int64_t(src.n) / 256 + 1, 8), 256, 0, st>>>(src.p, dst.p, int64_t(src.n));
        CK(cudaGetLastError());
    };
    std::shared_future<void> near_f = std::async(std::launch::async, [&]() {
        CK(cudaSetDevice(c->device));
        near_entries = build_near(c, s2, &h_ntoff);
        to_f32(c->N, c->N32, s2);
        to_f32(c->NT, c->NT32, s2);
        CK(cudaStreamSynchronize(s2));
        timer.mark("near field built");
    }).share();
    // The far pairs matched across the two sides' directional plans (which items a pair couples,
    // where its transpose sits) need the plans only: matched on a thread of their own while the
    // sides compress. The couplings then only add the ranks.
    std::promise<void> planned[2];
    std::shared_future<void> planned_f[2] = {planned[0].get_future().share(), planned[1].get_future().share()};
    std::vector<int32_t> pair_it, pair_is, pair_of_pos;
    std::shared_future<void> pairs_f = std::async(std::launch::async, [&]() {
        planned_f[0].get();
        planned_f[1].get();
        const nca::DirSide &pt = D->side[0].plan, &ps = D->side[1].plan;
        // far pairs (test CSR grouped by test direction) and their items on both sides
        std::vector<int32_t> item_of_pos[2];
        for (int sd = 0; sd < 2; ++sd) {
            const nca::DirSide &pl = D->side[sd].plan;
            item_of_pos[sd].assign(pl.farnodes.size(), -1);
            for (size_t it = 0; it < pl.item_node.size(); ++it)
                for (int q = pl.dirfarptr[it]; q < pl.dirfarptr[it + 1]; ++q) item_of_pos[sd][q] = int32_t(it);
        }
        // (trial node, test node) -> position in the trial far lists: each trial node's list sorted by
        // test node and searched by bisection
        std::vector<std::pair<int32_t, int32_t>> bytest(ps.farnodes.size());
        for (int sn = 0; sn < c->tree[1].nnodes; ++sn) {
            for (int q = ps.farptr[sn]; q < ps.farptr[sn + 1]; ++q) bytest[q] = {ps.farnodes[q], q};
            std::sort(bytest.begin() + ps.farptr[sn], bytest.begin() + ps.farptr[sn + 1]);
        }
        auto trialpos = [&](int sn, int t) {
            const auto b = bytest.begin() + ps.farptr[sn], e = bytest.begin() + ps.farptr[sn + 1];
            const auto it = std::lower_bound(b, e, std::make_pair(int32_t(t), INT32_MIN));
            if (it == e || it->first != t) throw Failure(NCA_ERR_ARG, "internal: a far pair has no transpose");
            return it->second;
        };
        const int64_t np = int64_t(pt.farnodes.size());
        pair_it.assign(np, 0);
        pair_is.assign(np, 0);
        pair_of_pos.assign(ps.farnodes.size(), -1);
        for (int t = 0; t < c->tree[0].nnodes; ++t)
            for (int e = pt.farptr[t]; e < pt.farptr[t + 1]; ++e) {
                const int sn = pt.farnodes[e];
                const int32_t q = trialpos(sn, t);
                pair_it[e] = item_of_pos[0][e];
                pair_is[e] = item_of_pos[1][q];
                pair_of_pos[q] = e;
            }
        timer.mark("far pairs matched");
    }).share();
    std::vector<std::vector<int32_t>> bylevel[2];  // items per level, filled by each side's task
    int64_t basis_entries[2] = {0, 0}, transfer_entries[2] = {0, 0};
    // a side's ranks, rows, operator offsets and coefficient offsets are known (side_ranked) before
    // its operators are joined and transposed on the device (side_done)
    std::promise<void> sided[2], ranked[2];
    std::shared_future<void> side_done[2] = {sided[0].get_future().share(), sided[1].get_future().share()};
    std::shared_future<void> side_ranked[2] = {ranked[0].get_future().share(), ranked[1].get_future().share()};
    std::atomic<bool> ranked_set[2] = {false, false};
    // Galerkin inputs (one tree on both sides, a symmetric partition) give the trial side the test
    // side's directional plan: it is made once and copied, instead of twice at once on the same
    // host cores
    const nca::Tree &T0 = c->tree[0], &T1 = c->tree[1];
    const bool symmetric = !sv && T0.nnodes == T1.nnodes && T0.perm == T1.perm && T0.begin == T1.begin &&
                           T0.end == T1.end && T0.parent == T1.parent && T0.firstchild == T1.firstchild &&
                           T0.nchildren == T1.nchildren && T0.level == T1.level && T0.center == T1.center &&
                           T0.radius == T1.radius && P.farptr == P.tfarptr && P.farnodes == P.tfarnodes;
    // ... and, when moreover both sides hold the same points, the kernel depends on |x - y| only
    // (Helmholtz, Laplace: K(x, y) and K(y, x) are formed from the same squared differences, bit for
    // bit) and the tolerances agree, the trial side's IACA would repeat the test side's bit for bit
    // (every entry, sum and pivot decision is the same): the trial side takes the test side's
    // ranks, pivots and operators (device copies) instead of a second compression.
    // NCA_MIRROR_TRIAL=0 compresses both sides.
    const bool mirror = [&] {
        const char *e = getenv("NCA_MIRROR_TRIAL");
        if (e && e[0] == '0') return false;
        return symmetric && (c->K.kind == 0 || c->K.kind == 1) && c->K.deriv == 0 && o->tol_test == o->tol_trial &&
               T0.npoints == T1.npoints &&
               std::memcmp(tp, sp, sizeof(double) * 3 * size_t(T0.npoints)) == 0;
    }();
    auto side_task = [&](int sd) {
        const cudaStream_t s = ss[sd];
        DirItems &d = D->side[sd];
        const std::string side = sd == 0 ? "test: " : "trial: ";
        try {
            if (sv) {
                d.plan = sv->side[sd].plan;
            } else if (symmetric && sd == 1) {
                planned_f[0].get();
                // member by member on threads of their own: the copy writes ~50 MB of fresh pages
                const nca::DirSide &src = D->side[0].plan;
                nca::DirSide &dst = d.plan;
                std::vector<std::future<void>> parts;
                auto copy = [&parts](auto &to, const auto &from) {
                    parts.push_back(std::async(std::launch::async, [&to, &from] { to = from; }));
                };
                copy(dst.farptr, src.farptr);
                copy(dst.farnodes, src.farnodes);
                copy(dst.dirptr, src.dirptr);
                copy(dst.dirs, src.dirs);
                copy(dst.dirvec, src.dirvec);
                copy(dst.dirfarptr, src.dirfarptr);
                copy(dst.chdirptr, src.chdirptr);
                copy(dst.chdirmap, src.chdirmap);
                copy(dst.invptr, src.invptr);
                copy(dst.invidx, src.invidx);
                copy(dst.item_node, src.item_node);
                copy(dst.item_basis, src.item_basis);
                copy(dst.item_chptr, src.item_chptr);
                copy(dst.item_chidx, src.item_chidx);
                for (auto &f : parts) f.get();
                static_assert(sizeof(nca::DirSide) == 14 * sizeof(std::vector<int32_t>),
                              "every member of DirSide is copied above");
            } else {
                d.plan = directional_plan(c->tree[sd], c->tree[1 - sd], sd == 0 ? P.farptr : P.tfarptr,
                                          sd == 0 ? P.farnodes : P.tfarnodes, wb);
            }
        } catch (...) {
            planned[sd].set_exception(std::current_exception());
            throw;
        }
        planned[sd].set_value();
        timer.mark(side + "directional plan (" + std::to_string(d.plan.item_node.size()) + " items)");
        const nca::DirSide &pl = d.plan;
        const nca::Tree &T = c->tree[sd];
        const int ni = int(pl.item_node.size());
        d.nitems = ni;
        bylevel[sd].assign(T.nlevels, {});
        for (int it = 0; it < ni; ++it) bylevel[sd][T.level[pl.item_node[it]]].push_back(it);
        auto known = [&]() {
            d.h_cptr.assign(ni + 1, 0);
            for (int it = 0; it < ni; ++it) {
                d.h_cptr[it + 1] = d.h_cptr[it] + d.h_rank[it];
                const int64_t e = int64_t(d.h_rank[it]) * d.h_nrows[it];
                (pl.item_basis[it] ? basis_entries[sd] : transfer_entries[sd]) += e;
            }
            ranked_set[sd] = true;
            ranked[sd].set_value();
            timer.mark(side + "ranks known");
        };
        if (sv) {
            // a saved skeleton: the items' operators and pivots as the build left them
            const SavedSide &v = sv->side[sd];
            d.item_node.upload(pl.item_node, s);
            d.item_basis.upload(pl.item_basis, s);
            d.item_chptr.upload(pl.item_chptr, s);
            d.item_chidx.upload(pl.item_chidx, s);
            d.rank.upload(v.rank, s);
            d.nrows.upload(v.nrows, s);
            d.piv.upload(v.piv, s);
            d.cpiv.upload(v.cpiv, s);
            d.h_rank = v.rank;
            d.h_nrows = v.nrows;
            d.h_xoff = v.xoff;
            known();
            d.X.upload(v.X, s);
        } else if (mirror && sd == 1) {
            // the test side's ranks and pivots are final once its ranks are known: copied before
            // this side's ranks are announced (the couplings read them on the device)
            side_ranked[0].get();
            const DirItems &d0 = D->side[0];
            auto dup = [&](auto &to, const auto &from) {
                to.alloc(from.n);
                if (from.n) CK(cudaMemcpyAsync(to.p, from.p, sizeof(*from.p) * from.n, cudaMemcpyDeviceToDevice, s));
            };
            dup(d.item_node, d0.item_node);
            dup(d.item_basis, d0.item_basis);
            dup(d.item_chptr, d0.item_chptr);
            dup(d.item_chidx, d0.item_chidx);
            dup(d.rank, d0.rank);
            dup(d.nrows, d0.nrows);
            dup(d.piv, d0.piv);
            dup(d.cpiv, d0.cpiv);
            CK(cudaStreamSynchronize(s));
            d.h_rank = d0.h_rank;
            d.h_nrows = d0.h_nrows;
            d.h_xoff = d0.h_xoff;
            known();
            side_done[0].get();  // the test side's operators are joined and transposed
            dup(d.xoff, d0.xoff);
            dup(d.X, d0.X);
            d.XT.alloc_scratch(d0.XT.n);
            if (d0.XT.n)
                CK(cudaMemcpyAsync(d.XT.p, d0.XT.p, sizeof(double2) * d0.XT.n, cudaMemcpyDeviceToDevice, s));
            CK(cudaStreamSynchronize(s));
            timer.mark(side + "operators taken from the test side");
            return;
        } else {
            compress_dir_side(c, d, sd, pts[sd], bylevel[sd], s, o, timer, side, known, hs[sd]);
        }
        d.xoff.upload(d.h_xoff, s);
        d.XT.alloc_scratch(d.X.n);
        launch_transpose_blocks<double2>(d.X.p, d.xoff.p, d.nrows.p, d.rank.p, d.xoff.p, ni, d.XT.p, s);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(s));
        timer.mark(side + "bases joined and transposed");
        };
    // couplings: computed by the thread of the forward coupling plan (the transposed coupling plan
    // waits for it) on stream s while the other plans are built; their device inputs stay alive
    // until s is synchronised
    const nca::DirSide &pt = D->side[0].plan, &ps = D->side[1].plan;
    int64_t npairs = 0;
    std::vector<int64_t> cfoff, ctoff;
    int64_t coupling_entries = 0;
    auto couplings = [&](cudaStream_t st) {
        npairs = int64_t(pt.farnodes.size());
        const std::vector<int32_t> &rt = D->side[0].h_rank, &rs = D->side[mirror ? 0 : 1].h_rank;
        // coupling blocks S_e = K[tau_(t, dt), tau_(s, ds)] in test pair order, transposes in trial order
        cfoff.assign(npairs + 1, 0);
        ctoff.assign(ps.farnodes.size() + 1, 0);
        for (int64_t e = 0; e < npairs; ++e) {
            const int64_t n = int64_t(rt[pair_it[e]]) * rs[pair_is[e]];
            coupling_entries += n;
            cfoff[e + 1] = cfoff[e] + pad2(n);
        }
        std::vector<int64_t> tr_in(ps.farnodes.size());
        std::vector<int32_t> tr_rows(ps.farnodes.size()), tr_cols(ps.farnodes.size());
        for (size_t q = 0; q < ps.farnodes.size(); ++q) {
            const int e = pair_of_pos[q];
            tr_in[q] = cfoff[e];
            tr_rows[q] = rt[pair_it[e]];
            tr_cols[q] = rs[pair_is[e]];
            ctoff[q + 1] = ctoff[q] + pad2(int64_t(tr_rows[q]) * tr_cols[q]);
        }
        // a mirrored core whose transposed block at every trial position is the forward block at
        // the same test position (the partners swap places and the offsets agree) shares the
        // forward coupling stage: the blocks are equal entry for entry (one point set, K(x, y) =
        // K(y, x) bit for bit, the same pivots on both sides)
        bool share = mirror && ctoff == cfoff;
        for (size_t q = 0; share && q < ps.farnodes.size(); ++q) {
            const int e = pair_of_pos[q];
            share = pair_is[e] == pair_it[q] && pair_it[e] == pair_is[q];
        }
        D->prod[1].same_couple = share;
        GatherStage &CN = D->prod[0].couple, &CTs = D->prod[1].couple;
        CN.M.alloc(size_t(cfoff.back()));
        if (!share) CTs.M.alloc(size_t(ctoff.back()));
        CN.entries = CTs.entries = coupling_entries;
        {
            // staged through page-locked memory on the coupling plan's stream (not behind the test
            // side's work on the build stream)
            {
                StagedUploads up(sizeof(int32_t) * (pair_it.size() + pair_is.size() + tr_rows.size() + tr_cols.size()) +
                                     sizeof(int64_t) * (cfoff.size() + tr_in.size() + ctoff.size()) + 8 * 16,
                                 st);
                up.up(D->cpair_it, pair_it);
                up.up(D->cpair_is, pair_is);
                up.up(D->ccoff, cfoff);
                up.up(D->ctr_in, tr_in);
                up.up(D->ctr_rows, tr_rows);
                up.up(D->ctr_cols, tr_cols);
                up.up(D->ctr_off, ctoff);
            }  // the copies have landed (the staging block goes back to the pool)
            D->npairs = npairs;
            CouplingArgs a;
            a.K = c->K;
            a.test_pts = c->side[0].pts.p;
            a.trial_pts = c->side[1].pts.p;
            a.pair_t = D->cpair_it.p;
            a.pair_s = D->cpair_is.p;
            a.rank_t = D->side[0].rank.p;
            a.rank_s = D->side[mirror ? 0 : 1].rank.p;
            a.piv_t = D->side[0].piv.p;
            a.piv_s = D->side[mirror ? 0 : 1].piv.p;
            a.maxrank = maxrank;
            a.coff = D->ccoff.p;
            a.npairs = npairs;
            a.C = CN.M.p;
            a.C32 = nullptr;
            if (npairs > 0 && !(a.rank_t && a.rank_s && a.piv_t && a.piv_s && a.C))
                throw Failure(NCA_ERR_CUDA, "internal: the couplings were reached before both sides' pivots");
            if (npairs > 0) {
                k_couplings<<<launch_grid(npairs, 16), 256, 0, st>>>(a);
                CK(cudaGetLastError());
            }
            D->ntr = share ? 0 : int64_t(ps.farnodes.size());  // no transposes when the stage is shared
            launch_transpose_blocks<double2>(CN.M.p, D->ctr_in.p, D->ctr_rows.p, D->ctr_cols.p, D->ctr_off.p, D->ntr,
                                             CTs.M.p, st);
            CK(cudaGetLastError());
            to_f32(CN.M, CN.M32, st);
            if (!share) to_f32(CTs.M, CTs.M32, st);
        }
    };
    std::promise<void> coupled;
    std::shared_future<void> coupled_done = coupled.get_future().share();
    cudaStream_t ts[8];
    for (cudaStream_t &t : ts) CK(cudaStreamCreateWithFlags(&t, cudaStreamNonBlocking));
    struct StreamsGuard {
        cudaStream_t *t;
        ~StreamsGuard() {
            for (int i = 0; i < 8; ++i) cudaStreamDestroy(t[i]);
        }
    } tsg{ts};
    auto plan_task = [&](int task) {
        const cudaStream_t s = ts[task];
        auto plan_mark = [&timer, task](const char *stage) {
            return [&timer, task, stage](const std::string &what) {
                timer.mark("gather plan " + std::to_string(task) + ": " + stage + " " + what);
            };
        };
        const int m = task / 4, stage = task % 4;
        const int I = m == 0 ? 1 : 0, O = 1 - I;
        // the sides whose host arrays (ranks, offsets, items) the plan reads: a mirrored trial
        // side's are the test side's, read from there as soon as the test side's ranks are known
        const int hI = mirror ? 0 : I, hO = mirror ? 0 : O;
        const DirItems &di = D->side[hI], &dout = D->side[hO];
        const nca::Tree &TI = c->tree[I], &TO = c->tree[O];
        DirProduct &pr = D->prod[m];
        if (pr.same && stage != 1) return;  // the forward product's stage serves this one
        // arena rows: [x of the input side; its coefficients; the output side's coefficients]: the
        // output rows start after the input side's coefficients, known once that side is built
        const int64_t xin = TI.npoints;
        int64_t yo = 0;
        auto input_side_built = [&]() {
            side_ranked[hI].get();
            yo = xin + di.h_cptr.back();
        };
        // up: input-side items, deepest level first
        if (stage == 0) {
            side_ranked[hI].get();
            StageBuilder B;
            const size_t seg = size_t(di.nitems) + di.plan.item_chidx.size();
            B.reserve(size_t(di.nitems), seg, seg);
            for (int lev = TI.nlevels - 1; lev >= 0; --lev) {
                for (int it : bylevel[hI][lev]) {
                    const int r = di.h_rank[it];
                    if (r <= 0) continue;
                    B.begin_output(r, xin + di.h_cptr[it]);
                    if (di.plan.item_basis[it]) {
                        const int node = di.plan.item_node[it];
                        const int nr = di.h_nrows[it];
                        B.segment(B.copy(di.h_xoff[it], r, r, nr), nr, TI.begin[node]);
                    } else {
                        int64_t c0 = 0;
                        for (int k = di.plan.item_chptr[it]; k < di.plan.item_chptr[it + 1]; ++k) {
                            const int ch = di.plan.item_chidx[k];
                            const int rc = di.h_rank[ch];
                            if (rc > 0) B.segment(B.copy(di.h_xoff[it] + c0 * r, r, r, rc), rc, xin + di.h_cptr[ch]);
                            c0 += rc;
                        }
                    }
                    B.end_output();
                }
                B.end_group();
            }
            timer.mark("gather plan " + std::to_string(task) + ": up listed");
            side_done[hI].get();
            B.finish(pr.up, di.XT.p, s, m ? "T up" : "N up", plan_mark("up"));
            to_f32(pr.up.M, pr.up.M32, s);
            timer.mark("gather plan " + std::to_string(task) + ": up");
        }
        // coupling: output-side items with a rank and their far pairs' blocks (store built above)
        if (stage == 1) {
            if (m == 0) {
                // every way out of this block settles `coupled`, which the transposed plan awaits
                try {
                    side_ranked[hO].get();
                    input_side_built();
                    pairs_f.get();
                    timer.mark("gather plan " + std::to_string(task) + ": couplings started");
                    couplings(s);
                    timer.mark("gather plan " + std::to_string(task) + ": couplings enqueued");
                    coupled.set_value();
                } catch (...) {
                    coupled.set_exception(std::current_exception());
                    throw;
                }
            } else {
                coupled_done.get();
                if (pr.same_couple) return;  // the forward coupling stage serves this product
                side_ranked[hO].get();
                input_side_built();
            }
            StageBuilder B;
            const nca::DirSide &pl = dout.plan;
            const std::vector<int64_t> &off = m == 0 ? cfoff : ctoff;
            B.reserve(size_t(dout.nitems), pl.farnodes.size(), 0);
            for (int it = 0; it < dout.nitems; ++it) {
                const int r = dout.h_rank[it];
                if (r <= 0) continue;
                B.begin_output(r, yo + dout.h_cptr[it]);
                for (int q = pl.dirfarptr[it]; q < pl.dirfarptr[it + 1]; ++q) {
                    const int e = m == 0 ? q : pair_of_pos[q];
                    const int other = m == 0 ? pair_is[e] : pair_it[e];
                    const int ro = di.h_rank[other];
                    if (ro > 0) B.segment(off[q], ro, xin + di.h_cptr[other]);
                }
                B.end_output();
            }
            B.end_group();
            timer.mark("gather plan " + std::to_string(task) + ": coupling listed");
            B.finish(pr.couple, nullptr, s, m ? "T coupling" : "N coupling", plan_mark("coupling"));
            timer.mark("gather plan " + std::to_string(task) + ": coupling");
        }
        // down: output-side items gather from the parent items that map onto them, root level first
        if (stage == 2) {
            // listed with output rows relative to yo (the other side may still be compressing),
            // moved by yo once it is known
            side_ranked[hO].get();
            // parents of every child item (CSR in parent order), with the child's row offset in
            // the parent's X
            hvec<int32_t> pptr(size_t(dout.nitems) + 1, 0), ppar;
            hvec<int64_t> prow;
            auto each_child = [&](auto fn) {
                for (int it = 0; it < dout.nitems; ++it) {
                    if (dout.h_rank[it] <= 0 || dout.plan.item_basis[it]) continue;
                    int64_t c0 = 0;
                    for (int k = dout.plan.item_chptr[it]; k < dout.plan.item_chptr[it + 1]; ++k) {
                        const int ch = dout.plan.item_chidx[k];
                        if (dout.h_rank[ch] > 0) fn(ch, it, c0);
                        c0 += dout.h_rank[ch];
                    }
                }
            };
            each_child([&](int ch, int, int64_t) { ++pptr[size_t(ch) + 1]; });
            for (int it = 0; it < dout.nitems; ++it) pptr[size_t(it) + 1] += pptr[it];
            ppar.resize(pptr.back());
            prow.resize(pptr.back());
            hvec<int32_t> fill(pptr.begin(), pptr.end() - 1);
            each_child([&](int ch, int it, int64_t c0) {
                ppar[fill[ch]] = it;
                prow[fill[ch]++] = c0;
            });
            StageBuilder B;
            B.reserve(size_t(dout.nitems), ppar.size(), ppar.size());
            for (int lev = 1; lev < TO.nlevels; ++lev) {
                for (int it : bylevel[hO][lev]) {
                    const int r = dout.h_rank[it];
                    if (r <= 0 || pptr[it + 1] == pptr[it]) continue;
                    B.begin_output(r, yo + dout.h_cptr[it]);
                    for (int q = pptr[it]; q < pptr[it + 1]; ++q) {
                        const int p = ppar[q];
                        const int rp = dout.h_rank[p];
                        B.segment(B.copy(dout.h_xoff[p] + prow[q], dout.h_nrows[p], r, rp), rp, yo + dout.h_cptr[p]);
                    }
                    B.end_output();
                }
                B.end_group();
            }
            timer.mark("gather plan " + std::to_string(task) + ": down listed");
            input_side_built();
            B.shift(yo, true);
            side_done[hO].get();
            B.finish(pr.down, dout.X.p, s, m ? "T down" : "N down", plan_mark("down"));
            to_f32(pr.down.M, pr.down.M32, s);
            timer.mark("gather plan " + std::to_string(task) + ": down");
        }
        // leaves: every basis item whose cluster contains the leaf, then the near blocks
        if (stage == 3) {
            side_ranked[hO].get();
            near_f.get();
            StageBuilder B;
            const nca::DirSide &pl = dout.plan;
            const std::vector<int32_t> &nptr = m == 0 ? P.nearptr : P.tnearptr;
            const std::vector<int32_t> &nnodes = m == 0 ? P.nearnodes : P.tnearnodes;
            for (int leaf = 0; leaf < TO.nnodes; ++leaf) {
                if (!TO.isleaf(leaf)) continue;
                const int R = TO.size(leaf);
                B.begin_output(R, TO.begin[leaf]);
                for (int a = leaf; a >= 0; a = TO.parent[a])
                    for (int it = pl.dirptr[a]; it < pl.dirptr[a + 1]; ++it) {
                        const int r = dout.h_rank[it];
                        if (r <= 0 || !pl.item_basis[it]) continue;
                        B.segment(B.copy(dout.h_xoff[it] + (TO.begin[leaf] - TO.begin[a]), dout.h_nrows[it], R, r), r,
                                  yo + dout.h_cptr[it]);
                    }
                for (int i = nptr[leaf]; i < nptr[leaf + 1]; ++i) {
                    const int other = nnodes[i];
                    const int64_t noff = m == 0 ? c->h_nfoff[i] : h_ntoff[i];
                    B.segment(-1 - noff, TI.size(other), TI.begin[other]);
                }
                B.end_output();
            }
            B.end_group();
            timer.mark("gather plan " + std::to_string(task) + ": leaves listed");
            input_side_built();
            B.shift(yo, false);
            side_done[hO].get();
            B.finish(pr.leaves, dout.X.p, s, m ? "T leaves" : "N leaves", plan_mark("leaves"));
            to_f32(pr.leaves.M, pr.leaves.M32, s);
            timer.mark("gather plan " + std::to_string(task) + ": leaves");
        }
        CK(cudaStreamSynchronize(s));
        };
    // The two sides (direction plan, far fields, IACA levels) and the eight gather plans (four
    // stages x two orientations) on ten host threads and streams: a plan starts as soon as the
    // sides it reads are built (up: the input side; down, leaves: the output side, then the input
    // side's coefficient count; coupling: both sides and the couplings).
    if (mirror) D->prod[1].same = &D->prod[0];
    on_threads(c->device, 10, [&](int task) {
        if (task < 2) {
            try {
                side_task(task);
            } catch (...) {
                if (!ranked_set[task]) ranked[task].set_exception(std::current_exception());
                sided[task].set_exception(std::current_exception());
                throw;
            }
            sided[task].set_value();
        } else {
            plan_task(task - 2);
        }
    });
    auto h1 = std::chrono::steady_clock::now();
    for (int m = 0; m < 2; ++m) {
        const int I = m == 0 ? 1 : 0, O = 1 - I;
        DirProduct &pr = D->prod[m];
        pr.nin = c->tree[I].npoints;
        pr.nout = c->tree[O].npoints;
        pr.cin = D->side[I].h_cptr.back();
        pr.cout = D->side[O].h_cptr.back();
    }
    CK(cudaStreamSynchronize(s));
    timer.mark("gather plans done");
    // the stage stores hold the products' copies of the operators; X stays for nca_core_save
    for (DirItems &d : D->side) d.XT.release();
    timer.mark("transposed bases released");
    CK(cudaEventRecord(ev1, s));
    CK(cudaStreamSynchronize(s));
    timer.mark("build complete");
    for (DirItems &d : D->side) d.free_later();
    timer.mark("scratch freed");
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ev0, ev1));
    auto h2 = std::chrono::steady_clock::now();
    nca_core_info &I = c->info;
    I.ntest = c->tree[0].npoints;
    I.ntrial = c->tree[1].npoints;
    I.nnodes_test = c->tree[0].nnodes;
    I.nnodes_trial = c->tree[1].nnodes;
    I.ncoeff_test = D->side[0].h_cptr.back();
    I.ncoeff_trial = D->side[1].h_cptr.back();
    I.near_entries = near_entries;
    I.coupling_entries = coupling_entries;
    I.basis_entries_test = basis_entries[0];
    I.basis_entries_trial = basis_entries[1];
    I.transfer_entries_test = transfer_entries[0];
    I.transfer_entries_trial = transfer_entries[1];
    I.nfarpairs = npairs;
    I.nnearpairs = int64_t(P.nearnodes.size());
    I.build_seconds = ms * 1e-3;
    I.build_seconds_host = std::chrono::duration<double>(h1 - h0).count() +
                           std::chrono::duration<double>(h2 - h1).count() - ms * 1e-3;
    c->dir = std::move(D);
}

// Device buffers one product runs on: the gathered input (nin x vs), the input side's
// coefficients xhat and the output side's yhat (coefficient rows x vs), and the error word the
// kernels raise (must be zero when the product starts).
struct ProductBuffers {
    double2 *xt, *xhat, *yhat;
    int32_t *error;
    bool far, near;
};

// Records a timing event; inside a stream capture as an external event node, so that the event
// is recorded each time the graph runs.
cudaError_t record_stage_event(cudaEvent_t ev, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cs);
    if (e != cudaSuccess) return e;
    return cudaEventRecordWithFlags(ev, st, cs == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : 0);
}

// Launch counts of one product: total and per stage (gather, up, couple, down, near field,
// leaves).
constexpr int kStages = 6;
struct ProductLaunches {
    int total = 0;
    int stage[kStages] = {0, 0, 0, 0, 0, 0};
};

// Stage events of one product (profiling): the gather, the three far-field sweeps on the sweep
// stream, the near field and the leaf stage on the product stream.
enum StageEvent { EV_START, EV_GATHER, EV_UP, EV_COUPLE, EV_DOWN, EV_NEAR0, EV_NEAR1, EV_LEAVES0, EV_END, EV_COUNT };

// Second stream of a product: with aux set, the far-field sweeps (upward, coupling, downward)
// run on aux while the near field streams on the product stream; fork and join order them.
struct ProductStreams {
    cudaStream_t aux = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    int priority = 0;  // the sweeps' launch priority (that of aux)
};

// Enqueues the gather and the product stages of y = alpha op(A) x + beta y on stream s. x, y are
// device arrays (ldx, ldy leading dimensions); stage_ev (nullable) receives EV_COUNT events.
//
// Serial form (no aux stream): per 16-column pass, upward sweep, coupling, downward sweep and one
// leaf launch y_t = alpha (X_t yhat_t + sum_s N_ts x_s) + beta y_t.
// Overlapped form (aux stream, far and near parts): the near field depends on the gathered x
// alone, so it runs beside the sweeps: y_t = alpha sum_s N_ts x_s + beta y_t on s while aux runs
// the sweeps; after the join a leaf-basis launch adds alpha X_t yhat_t. The near field is the
// bandwidth-bound bulk of the product and the sweeps are chains of small launches per tree
// level, so the sweeps' latency hides under the near field's streaming. Results differ from the
// serial form only in the rounding of the final sum.
int enqueue_product(nca_core *c, int mode, int precision, const double2 *xd, int64_t lx, double2 *yd,
                    int64_t ly, int b, double2 alpha, double2 beta, const ProductBuffers &buf,
                    cudaStream_t s, cudaEvent_t *stage_ev, ProductLaunches &count,
                    const ProductStreams &ps = ProductStreams{}) {
    const int in = mode == 0 ? 1 : 0, out = 1 - in;
    const int64_t nin = c->side[in].npts;
    DevSide &I = c->side[in], &O = c->side[out];
    const int vs = vector_stride(b);
    const bool usebeta = beta.x != 0.0 || beta.y != 0.0;
    const int cap = rows_capacity(std::min(b, 16));
    if (O.leafcap > cap || I.leafcap > cap || 2 * c->maxrank > cap)
        return fail(NCA_ERR_ARG, "a leaf or transfer block has more rows than one product CTA holds");
    const bool overlap = ps.aux != nullptr && buf.far && buf.near;
    auto mark = [&](int k, cudaStream_t st) {
        if (stage_ev) CK(record_stage_event(stage_ev[k], st));
    };
    mark(EV_START, s);
    k_gather<<<launch_grid(nin * b / 256 + 1, 8), 256, 0, s>>>(xd, lx, I.perm.p, nin, b, vs, buf.xt);
    ++count.total;
    ++count.stage[0];
    mark(EV_GATHER, s);
    const bool conj = mode == 2;
    auto run = [&](auto tag) {
        using S = decltype(tag);
        constexpr bool f64 = std::is_same<S, double2>::value;
        const S *XTi = f64 ? (const S *)I.XT.p : (const S *)I.XT32.p;
        const S *Xo = f64 ? (const S *)O.X.p : (const S *)O.X32.p;
        const S *Cm = nullptr, *Nm = nullptr;
        if (mode == 0) {
            Cm = f64 ? (const S *)c->C.p : (const S *)c->C32.p;
            Nm = f64 ? (const S *)c->N.p : (const S *)c->N32.p;
        } else {
            Cm = f64 ? (const S *)c->CT.p : (const S *)c->CT32.p;
            Nm = f64 ? (const S *)c->NT.p : (const S *)c->NT32.p;
        }
        // far-field sweeps of one 16-column pass on stream st: the upward sweep (with up) and the
        // coupling and downward sweep (with rest)
        auto sweeps = [&](int q0, int bc, cudaStream_t st, bool first, bool up, bool rest) {
            // upward sweep: xhat_p = XT_p [leaf x slice | children's xhat], deepest level first
            for (size_t l = 0; up && l + 1 < I.up.ptr.size(); ++l) {
                const int cnt = I.up.ptr[l + 1] - I.up.ptr[l];
                if (!cnt) continue;
                RowArgs<S> a{};
                a.stage = STAGE_UP;
                a.begin = I.begin.p;
                a.firstchild = I.firstchild.p;
                a.nchildren = I.nchildren.p;
                a.rank = I.rank.p;
                a.nrows = I.nrows.p;
                a.cptr = I.cptr.p;
                a.M = XTi;
                a.moff = I.xoff.p;
                a.src = buf.xt;
                a.coef = buf.xhat;
                a.b = b;
                a.bc = bc;
                a.q0 = q0;
                a.vs = vs;
                a.conj = conj && in == 0;
                a.maxrows = I.up.mcap[l];
                a.error = buf.error;
                launch_rows<S>(a, I.up.d_nodes.p + I.up.ptr[l], cnt, st, 0, st == ps.aux ? ps.priority : 0);
                ++count.total;
                ++count.stage[1];
            }
            if (first && up) mark(EV_UP, st);
            if (!rest) return;
            const int ncp = mode == 0 ? c->n_couple_fwd : c->n_couple_rev;
            if (ncp > 0) {
                RowArgs<S> a{};
                a.stage = STAGE_COUPLE;
                a.M = Cm;
                if (mode == 0) {
                    a.moff = c->cfoff.p;
                    a.ptr = c->farptr.p;
                    a.other = c->farnodes.p;
                } else {
                    a.moff = c->ctoff.p;
                    a.ptr = c->tfarptr.p;
                    a.other = c->tfarnodes.p;
                }
                a.rank_in = I.rank.p;
                a.rank_out = O.rank.p;
                a.cptr_in = I.cptr.p;
                a.cptr_out = O.cptr.p;
                a.src = buf.xhat;
                a.dst = buf.yhat;
                a.b = b;
                a.bc = bc;
                a.q0 = q0;
                a.vs = vs;
                a.conj = conj;
                a.maxrows = c->maxrank;
                a.error = buf.error;
                launch_rows<S>(a, mode == 0 ? c->couple_fwd.p : c->couple_rev.p, ncp, st, 0,
                               st == ps.aux ? ps.priority : 0);
                ++count.total;
                ++count.stage[2];
            }
            if (first) mark(EV_COUPLE, st);
            // downward sweep: [yhat_children] += X_p yhat_p, root level first
            for (size_t l = 0; l + 1 < O.down.ptr.size(); ++l) {
                const int cnt = O.down.ptr[l + 1] - O.down.ptr[l];
                if (!cnt) continue;
                RowArgs<S> a{};
                a.stage = STAGE_DOWN;
                a.firstchild = O.firstchild.p;
                a.rank = O.rank.p;
                a.nrows = O.nrows.p;
                a.cptr = O.cptr.p;
                a.M = Xo;
                a.moff = O.xoff.p;
                a.coef = buf.yhat;
                a.b = b;
                a.bc = bc;
                a.q0 = q0;
                a.vs = vs;
                a.conj = conj && out == 1;
                a.maxrows = O.down.mcap[l];
                a.error = buf.error;
                launch_rows<S>(a, O.down.d_nodes.p + O.down.ptr[l], cnt, st, 0, st == ps.aux ? ps.priority : 0);
                ++count.total;
                ++count.stage[3];
            }
            if (first) mark(EV_DOWN, st);
        };
        // leaf stage of one pass: y_t = al (X_t yhat_t [with_basis] + sum_s N_ts x_s [with_near]) + be y_t
        auto leaves = [&](int q0, int bc, bool with_basis, bool with_near, double2 al, double2 be, bool ube,
                          int stage) {
            RowArgs<S> a{};
            a.stage = STAGE_LEAVES;
            a.begin = O.begin.p;
            a.end = O.end.p;
            a.perm = O.perm.p;
            a.rank = O.rank.p;
            a.cptr = O.cptr.p;
            a.X = with_basis ? Xo : nullptr;
            a.xoff = O.xoff.p;
            a.coef = buf.yhat;
            if (with_near) {
                a.M = Nm;
                a.moff = mode == 0 ? c->nfoff.p : c->ntoff.p;
                a.ptr = mode == 0 ? c->nearptr.p : c->tnearptr.p;
                a.other = mode == 0 ? c->nearnodes.p : c->tnearnodes.p;
            }
            a.o_begin = I.begin.p;
            a.o_end = I.end.p;
            a.src = buf.xt;
            a.y = yd;
            a.ldy = ly;
            a.alpha = al;
            a.beta = be;
            a.usebeta = ube;
            a.b = b;
            a.bc = bc;
            a.q0 = q0;
            a.vs = vs;
            a.conj = conj;
            a.maxrows = O.leafcap;
            a.error = buf.error;
            launch_rows<S>(a, O.leaves.p, O.nleaves, s);
            ++count.total;
            ++count.stage[stage];
        };
        if (overlap) {
            // (forking after the upward sweep instead, so that it runs alone, measured 5 % slower:
            // the downward sweep's small launches then wait longer for SM slots)
            CK(cudaEventRecord(ps.fork, s));
            CK(cudaStreamWaitEvent(ps.aux, ps.fork, 0));
            for (int q0 = 0; q0 < b; q0 += 16) sweeps(q0, std::min(16, b - q0), ps.aux, q0 == 0, true, true);
            CK(cudaEventRecord(ps.join, ps.aux));
            mark(EV_NEAR0, s);
            for (int q0 = 0; q0 < b; q0 += 16) leaves(q0, std::min(16, b - q0), false, true, alpha, beta, usebeta, 4);
            mark(EV_NEAR1, s);
            CK(cudaStreamWaitEvent(s, ps.join, 0));
            mark(EV_LEAVES0, s);
            // y_t += alpha X_t yhat_t
            for (int q0 = 0; q0 < b; q0 += 16)
                leaves(q0, std::min(16, b - q0), true, false, alpha, make_double2(1.0, 0.0), true, 5);
        } else {
            for (int q0 = 0; q0 < b; q0 += 16) {
                const int bc = std::min(16, b - q0);
                if (buf.far) sweeps(q0, bc, s, q0 == 0, true, true);
                if (q0 == 0) {
                    if (!buf.far) {
                        mark(EV_UP, s);
                        mark(EV_COUPLE, s);
                        mark(EV_DOWN, s);
                    }
                    mark(EV_NEAR0, s);
                    mark(EV_NEAR1, s);
                    mark(EV_LEAVES0, s);
                }
                leaves(q0, bc, buf.far, buf.near, alpha, beta, usebeta, 5);
            }
        }
        mark(EV_END, s);
    };
    if (precision == NCA_PREC_F64)
        run(double2{});
    else
        run(float2{});
    CK(cudaGetLastError());
    return NCA_OK;
}

// Enqueues y = alpha (dH/dk) x + beta y (forward mode, complex FP64) on the frozen skeleton:
// the product's sweeps carried as dual numbers (xhat, dxhat) and (yhat, dyhat):
//   up       xhat_p = X_p^T src_p,   dxhat_p = dX_p^T src_p + X_p^T dxhat_children
//   coupling yhat = S xhat,          dyhat = S dxhat + dS xhat
//   down     yhat_c += X_p yhat_p,   dyhat_c += X_p dyhat_p + dX_p yhat_p
//   leaves   dy_t = X_t dyhat_t + dX_t yhat_t + sum_s dN_ts x_s
// dxhat and dyhat have the shapes of xhat and yhat.
int enqueue_tangent(nca_core *c, const double2 *xd, int64_t lx, double2 *yd, int64_t ly, int b, double2 alpha,
                    double2 beta, const ProductBuffers &buf, double2 *dxhat, double2 *dyhat, cudaStream_t s,
                    ProductLaunches &count) {
    DevSide &I = c->side[1], &O = c->side[0];
    const int64_t nin = I.npts;
    const int vs = vector_stride(b);
    const int cap = rows_capacity(std::min(b, 16));
    if (O.leafcap > cap || I.leafcap > cap || 2 * c->maxrank > cap)
        return fail(NCA_ERR_ARG, "a leaf or transfer block has more rows than one product CTA holds");
    k_gather<<<launch_grid(nin * b / 256 + 1, 8), 256, 0, s>>>(xd, lx, I.perm.p, nin, b, vs, buf.xt);
    ++count.total;
    auto go = [&](RowArgs<double2> &a, const int32_t *nodes, int cnt) {
        a.error = buf.error;
        a.b = b;
        a.vs = vs;
        launch_rows<double2>(a, nodes, cnt, s);
        ++count.total;
    };
    for (int q0 = 0; q0 < b; q0 += 16) {
        const int bc = std::min(16, b - q0);
        for (size_t l = 0; l + 1 < I.up.ptr.size(); ++l) {
            const int cnt = I.up.ptr[l + 1] - I.up.ptr[l];
            if (!cnt) continue;
            const int32_t *nodes = I.up.d_nodes.p + I.up.ptr[l];
            for (int pass = 0; pass < 3; ++pass) {
                RowArgs<double2> a{};
                a.stage = STAGE_UP;
                a.begin = I.begin.p;
                a.firstchild = I.firstchild.p;
                a.nchildren = I.nchildren.p;
                a.rank = I.rank.p;
                a.nrows = I.nrows.p;
                a.cptr = I.cptr.p;
                a.moff = I.xoff.p;
                a.src = buf.xt;
                a.bc = bc;
                a.q0 = q0;
                a.maxrows = I.up.mcap[l];
                if (pass == 0) {  // xhat_p = X_p^T src
                    a.M = I.XT.p;
                    a.coef = buf.xhat;
                } else if (pass == 1) {  // dxhat_p = dX_p^T src
                    a.M = I.dXT.p;
                    a.coef = buf.xhat;
                    a.coef_out = dxhat;
                } else {  // dxhat_p += X_p^T dxhat_children
                    a.M = I.XT.p;
                    a.coef = dxhat;
                    a.accumulate = 1;
                    a.skip_leaves = 1;
                }
                go(a, nodes, cnt);
            }
        }
        const int ncp = c->n_couple_fwd;
        if (ncp > 0)
            for (int pass = 0; pass < 3; ++pass) {
                RowArgs<double2> a{};
                a.stage = STAGE_COUPLE;
                a.M = pass == 2 ? c->dC.p : c->C.p;
                a.moff = c->cfoff.p;
                a.ptr = c->farptr.p;
                a.other = c->farnodes.p;
                a.rank_in = I.rank.p;
                a.rank_out = O.rank.p;
                a.cptr_in = I.cptr.p;
                a.cptr_out = O.cptr.p;
                a.src = pass == 1 ? dxhat : buf.xhat;
                a.dst = pass == 0 ? buf.yhat : dyhat;
                a.accumulate = pass == 2;
                a.bc = bc;
                a.q0 = q0;
                a.maxrows = c->maxrank;
                go(a, c->couple_fwd.p, ncp);
            }
        for (size_t l = 0; l + 1 < O.down.ptr.size(); ++l) {
            const int cnt = O.down.ptr[l + 1] - O.down.ptr[l];
            if (!cnt) continue;
            for (int pass = 0; pass < 3; ++pass) {
                RowArgs<double2> a{};
                a.stage = STAGE_DOWN;
                a.firstchild = O.firstchild.p;
                a.rank = O.rank.p;
                a.nrows = O.nrows.p;
                a.cptr = O.cptr.p;
                a.moff = O.xoff.p;
                a.M = pass == 2 ? O.dX.p : O.X.p;
                a.coef = pass == 1 ? dyhat : buf.yhat;
                a.coef_out = pass == 2 ? dyhat : nullptr;
                a.bc = bc;
                a.q0 = q0;
                a.maxrows = O.down.mcap[l];
                go(a, O.down.d_nodes.p + O.down.ptr[l], cnt);
            }
        }
        for (int pass = 0; pass < 2; ++pass) {
            RowArgs<double2> a{};
            a.stage = STAGE_LEAVES;
            a.begin = O.begin.p;
            a.end = O.end.p;
            a.perm = O.perm.p;
            a.rank = O.rank.p;
            a.cptr = O.cptr.p;
            a.xoff = O.xoff.p;
            a.o_begin = I.begin.p;
            a.o_end = I.end.p;
            a.src = buf.xt;
            a.y = yd;
            a.ldy = ly;
            a.alpha = alpha;
            if (pass == 0) {  // y = alpha (X dyhat + dN x) + beta y
                a.X = O.X.p;
                a.coef = dyhat;
                a.M = c->dN.p;
                a.moff = c->nfoff.p;
                a.ptr = c->nearptr.p;
                a.other = c->nearnodes.p;
                a.beta = beta;
                a.usebeta = beta.x != 0.0 || beta.y != 0.0;
            } else {  // y += alpha dX yhat
                a.X = O.dX.p;
                a.coef = buf.yhat;
                a.beta = make_double2(1.0, 0.0);
                a.usebeta = 1;
            }
            a.bc = bc;
            a.q0 = q0;
            a.maxrows = O.leafcap;
            go(a, O.leaves.p, O.nleaves);
        }
    }
    CK(cudaGetLastError());
    return NCA_OK;
}

// Enqueues y = alpha op(H) x + beta y for a directional core: gather x into the arena, then the
// up, coupling, down and leaf gathers (mode C = mode T with every block conjugated).
// Stage timing of a directional product: an event pair around each stage launch sequence (the
// gather is stage 0, then up 1, coupling 2, down 3 and leaves 5, the near field being part of the
// leaf outputs); events are created as needed.
struct DirTimer {
    std::vector<cudaEvent_t> *ev;
    std::vector<int> *stage;
    void mark(int k, bool end, cudaStream_t s) {
        const size_t i = stage->size() * 2 + (end ? 1 : 0);
        while (ev->size() <= i) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            ev->push_back(e);
        }
        CK(cudaEventRecord((*ev)[i], s));
        if (end) stage->push_back(k);
    }
};

int enqueue_dir_product(nca_core *c, int mode, int precision, const double2 *xd, int64_t lx, double2 *yd,
                        int64_t ly, int b, double2 alpha, double2 beta, double2 *arena, int32_t *error,
                        cudaStream_t s, ProductLaunches &count, DirTimer *timer = nullptr) {
    DirProduct &pr = c->dir->prod[mode == 0 ? 0 : 1];
    const int I = mode == 0 ? 1 : 0, O = 1 - I;
    const int vs = vector_stride(b);
    const int cap = rows_capacity(std::min(b, 16));
    for (const GatherStage *G : {&pr.up_stage(), &pr.couple_stage(), &pr.down_stage(), &pr.leaf_stage()})
        for (int r : G->group_maxrows)
            if (r > cap) return fail(NCA_ERR_ARG, "a leaf or basis block has more rows than one product CTA holds");
    // Complex-FP32 products keep the arena [x; coefficients] in complex FP32 too: the stages
    // accumulate in FP64 and round each output row once, and the vector rows, which outweigh
    // the FP32 blocks of these tiny gathers, move half the bytes.
    float2 *arena32 = reinterpret_cast<float2 *>(arena);
    if (timer) timer->mark(0, false, s);
    if (precision == NCA_PREC_F64)
        k_gather<<<launch_grid(pr.nin * b / 256 + 1, 8), 256, 0, s>>>(xd, lx, c->side[I].perm.p, pr.nin, b, vs, arena);
    else
        k_gather_to_f32<<<launch_grid(pr.nin * b / 256 + 1, 8), 256, 0, s>>>(xd, lx, c->side[I].perm.p, pr.nin, b, vs,
                                                                             arena32);
    ++count.total;
    ++count.stage[0];
    if (timer) timer->mark(0, true, s);
    const bool conj = mode == 2;
    // Stage by stage (each stage's levels in order): a launch group of small outputs over complex
    // FP32 stores takes every right-hand side in one k_gather_wide launch; any other group runs
    // once per 16-column pass. A group depends only on earlier groups' outputs for the same
    // columns, so this order computes what the pass-major order computes.
    auto run = [&](auto tag) {
        using S = decltype(tag);
        constexpr bool f64 = std::is_same<S, double2>::value;
        using VT = S;  // FP64 stores with FP64 vectors, FP32 stores with FP32 vectors
        // a shared leaf stage lists the forward near blocks (the mirrored core's transpose is the
        // matrix itself)
        const bool fwd = mode == 0 || pr.same;
        const S *nearM = f64 ? (const S *)(fwd ? c->N.p : c->NT.p) : (const S *)(fwd ? c->N32.p : c->NT32.p);
        auto stage = [&](const GatherStage &G, bool accumulate, bool scatter, int sk) {
            const S *M = f64 ? (const S *)G.M.p : (const S *)G.M32.p;
            if (timer) timer->mark(sk, false, s);
            for (size_t g = 0; g + 1 < G.group_ptr.size(); ++g) {
                const int cnt = G.group_ptr[g + 1] - G.group_ptr[g];
                if (!cnt) continue;
                RowArgs<S> a{};
                a.stage = STAGE_GATHER;
                a.M = M;
                a.M2 = nearM;
                a.g_rows = G.rows.p;
                a.g_out = G.out.p;
                a.g_segptr = G.segptr.p;
                a.g_moff = G.moff.p;
                a.g_w = G.w.p;
                a.g_voff = G.voff.p;
                if (f64) {
                    a.src = arena;
                    a.dst = arena;
                } else {
                    a.src32 = arena32;
                    a.dst32 = arena32;
                }
                a.accumulate = accumulate;
                if (scatter) {
                    a.y = yd;
                    a.ldy = ly;
                    a.perm = c->side[O].perm.p;
                    a.alpha = alpha;
                    a.beta = beta;
                    a.usebeta = beta.x != 0.0 || beta.y != 0.0;
                }
                a.b = b;
                a.vs = vs;
                a.conj = conj;
                a.maxrows = G.group_maxrows[g];
                a.error = error;
                const bool small = G.group_work[g] < kSmallGroupWork;
                if constexpr (!f64) {
                    // groups of small outputs on the FP32 pipe (all columns per launch); larger
                    // outputs of many right-hand sides on the tensor cores
                    if (b >= kTensorCoreColumns && gather_tc_fits(a.maxrows) &&
                        !wide_group(a.maxrows, G.group_work[g])) {
                        launch_gather_tc(a, G.tout.p + G.group_ptr[g], cnt, s);
                        ++count.total;
                        ++count.stage[sk];
                        continue;
                    }
                    if (b >= 2 && wide_group(a.maxrows, G.group_work[g])) {
                        for (int32_t k = G.wide_gptr[g]; k < G.wide_gptr[g + 1]; ++k) {
                            launch_gather_wide(a, G.wout.p + G.wide_begin[k], G.wide_count[k], G.wide_nr[k], s);
                            ++count.total;
                            ++count.stage[sk];
                        }
                        continue;
                    }
                }
                for (int q0 = 0; q0 < b; q0 += 16) {
                    a.bc = std::min(16, b - q0);
                    a.q0 = q0;
                    // many small outputs: one warp streams a sequence of them (up to 32 rows) or
                    // takes one (up to 64 rows); few large ones: the streaming MMA kernel
                    if (small && gather_tiny_fits(a.maxrows, a.bc))
                        launch_gather_tiny<S, VT>(a, G.outputs.p + G.group_ptr[g], cnt, s);
                    else if (a.maxrows <= 64 && small)
                        launch_gather_small<S, VT>(a, G.outputs.p + G.group_ptr[g], cnt, s);
                    else
                        launch_gather_rows<S, VT>(a, G.outputs.p + G.group_ptr[g], cnt, s);
                    ++count.total;
                    ++count.stage[sk];
                }
            }
            if (timer) timer->mark(sk, true, s);
        };
        stage(pr.up_stage(), false, false, 1);
        stage(pr.couple_stage(), false, false, 2);
        stage(pr.down_stage(), true, false, 3);
        stage(pr.leaf_stage(), false, true, 5);
    };
    if (precision == NCA_PREC_F64)
        run(double2{});
    else
        run(float2{});
    CK(cudaGetLastError());
    return NCA_OK;
}

// Tangent product of a directional core, dy = alpha (dH/dk) x + beta y on the frozen skeleton
// (forward mode, complex FP64): the four gather stages run on dual numbers. The arena holds two
// halves of R = nin + cin + cout rows: [x; x^; y^] and [0; dx^; dy^]; every stage computes its
// values in the first half and its derivative in the second as dM v + M dv (the second term reads
// the second half, whose x rows are zero, so the near blocks and the leaf bases' x slices drop out
// of it); the leaf stage writes dy = dL y^ + L dy^ (with dN x among dL y^).
int enqueue_dir_tangent(nca_core *c, const double2 *xd, int64_t lx, double2 *yd, int64_t ly, int b, double2 alpha,
                        double2 beta, double2 *arena, int32_t *error, cudaStream_t s, ProductLaunches &count) {
    DirProduct &pr = c->dir->prod[0];
    const int I = 1, O = 0;
    const int vs = vector_stride(b);
    const int cap = rows_capacity(std::min(b, 16));
    for (const GatherStage *G : {&pr.up, &pr.couple, &pr.down, &pr.leaves})
        for (int r : G->group_maxrows)
            if (r > cap) return fail(NCA_ERR_ARG, "a leaf or basis block has more rows than one product CTA holds");
    const int64_t R = pr.nin + pr.cin + pr.cout;
    double2 *A = arena, *B = arena + R * vs;
    k_gather<<<launch_grid(pr.nin * b / 256 + 1, 8), 256, 0, s>>>(xd, lx, c->side[I].perm.p, pr.nin, b, vs, A);
    CK(cudaMemsetAsync(B, 0, sizeof(double2) * size_t(pr.nin) * vs, s));
    ++count.total;
    const double2 *N = c->N.p, *dN = c->dN.p;
    for (int q0 = 0; q0 < b; q0 += 16) {
        const int bc = std::min(16, b - q0);
        auto group = [&](const GatherStage &G, size_t g, const double2 *M, const double2 *M2, double2 *src,
                         double2 *dst, bool accumulate, bool scatter, double2 bt) {
            const int cnt = G.group_ptr[g + 1] - G.group_ptr[g];
            if (!cnt) return;
            RowArgs<double2> a{};
            a.stage = STAGE_GATHER;
            a.M = M;
            a.M2 = M2;
            a.g_rows = G.rows.p;
            a.g_out = G.out.p;
            a.g_segptr = G.segptr.p;
            a.g_moff = G.moff.p;
            a.g_w = G.w.p;
            a.g_voff = G.voff.p;
            a.src = src;
            a.dst = dst;
            a.accumulate = accumulate;
            if (scatter) {
                a.y = yd;
                a.ldy = ly;
                a.perm = c->side[O].perm.p;
                a.alpha = alpha;
                a.beta = bt;
                a.usebeta = bt.x != 0.0 || bt.y != 0.0;
            }
            a.b = b;
            a.bc = bc;
            a.q0 = q0;
            a.vs = vs;
            a.conj = false;
            a.maxrows = G.group_maxrows[g];
            a.error = error;
            if (G.group_work[g] < kSmallGroupWork && gather_tiny_fits(a.maxrows, bc))
                launch_gather_tiny<double2, double2>(a, G.outputs.p + G.group_ptr[g], cnt, s);
            else if (a.maxrows <= 64 && G.group_work[g] < kSmallGroupWork)
                launch_gather_small<double2, double2>(a, G.outputs.p + G.group_ptr[g], cnt, s);
            else
                launch_gather_rows<double2, double2>(a, G.outputs.p + G.group_ptr[g], cnt, s);
            ++count.total;
        };
        // value, derivative of the store, store times derivative: level by level where levels depend
        auto dual = [&](const GatherStage &G, bool accumulate) {
            for (size_t g = 0; g + 1 < G.group_ptr.size(); ++g) {
                group(G, g, G.M.p, N, A, A, accumulate, false, beta);
                group(G, g, G.dM.p, dN, A, B, accumulate, false, beta);
                group(G, g, G.M.p, N, B, B, true, false, beta);
            }
        };
        dual(pr.up, false);
        dual(pr.couple, false);
        dual(pr.down, true);
        const double2 one = make_double2(1.0, 0.0);
        for (size_t g = 0; g + 1 < pr.leaves.group_ptr.size(); ++g) {
            group(pr.leaves, g, pr.leaves.dM.p, dN, A, nullptr, false, true, beta);
            group(pr.leaves, g, pr.leaves.M.p, N, B, nullptr, false, true, one);
        }
    }
    CK(cudaGetLastError());
    return NCA_OK;
}

// Argument checks shared by the product entry points.
int check_product_args(nca_core *c, int mode, int precision, int64_t ldx, int64_t ldy, int64_t nrhs) {
    if (mode < 0 || mode > 2) return fail(NCA_ERR_ARG, "mode must be 0 (N), 1 (T) or 2 (C)");
    if (precision != NCA_PREC_F64 && precision != NCA_PREC_F32) return fail(NCA_ERR_ARG, "unknown precision");
    if (precision == NCA_PREC_F32 && !c->f32)
        return fail(NCA_ERR_ARG, "complex FP32 product requested but the core was built without store_f32");
    const int in = mode == 0 ? 1 : 0, out = 1 - in;
    if (nrhs < 0 || ldx < c->side[in].npts || ldy < c->side[out].npts)
        return fail(NCA_ERR_DIM, "DimensionMismatch: leading dimension smaller than the operator size");
    return NCA_OK;
}

// Destroys the workspace's graphs and forgets the arguments seen (buffers are about to move).
void drop_graphs(nca_workspace *ws) {
    for (auto &g : ws->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    ws->graphs.clear();
    ws->seen.clear();
    ++ws->gen;
}

int apply_impl(nca_workspace *ws, int mode, int precision, const void *x, int64_t ldx, void *y,
               int64_t ldy, int64_t nrhs, double2 alpha, double2 beta, int memspace, bool tangent = false) {
    nca_core *c = ws->core;
    if (c->moved) return fail(NCA_ERR_ARG, "the core's stores were moved into a batch");
    if (int st = check_product_args(c, mode, precision, ldx, ldy, nrhs)) return st;
    if (tangent && (mode != 0 || precision != NCA_PREC_F64))
        return fail(NCA_ERR_ARG, "the d/dk product is forward mode and complex FP64");
    if (tangent && !c->has_dk) return fail(NCA_ERR_ARG, "call nca_core_prepare_dk before the d/dk product");
    const int in = mode == 0 ? 1 : 0, out = 1 - in;
    const int64_t nin = c->side[in].npts, nout = c->side[out].npts;
    if (nrhs == 0) return NCA_OK;
    CK(cudaSetDevice(c->device));
    cudaStream_t s = ws->stream;
    const int b = int(nrhs);
    if (b > ws->max_nrhs && !c->dir) {
        const int vsm = vector_slots(b);
        drop_graphs(ws);
        ws->xt.alloc(size_t(std::max(c->side[0].npts, c->side[1].npts)) * vsm);
        ws->xhat.alloc(size_t(std::max(c->side[0].h_cptr.back(), c->side[1].h_cptr.back())) * vsm);
        ws->yhat.alloc(ws->xhat.n);
        ws->max_nrhs = b;
    }
    const double2 *xd = reinterpret_cast<const double2 *>(x);
    double2 *yd = reinterpret_cast<double2 *>(y);
    int64_t lx = ldx, ly = ldy;
    const bool usebeta = beta.x != 0.0 || beta.y != 0.0;
    if (memspace == 0) {
        if (ws->xstage.n < size_t(nin) * b) ws->xstage.alloc(size_t(nin) * b);
        if (ws->ystage.n < size_t(nout) * b) ws->ystage.alloc(size_t(nout) * b);
    }
    CK(cudaEventRecord(ws->e0, s));
    CK(cudaMemsetAsync(ws->error.p, 0, sizeof(int32_t), s));
    if (memspace == 0) {
        CK(cudaMemcpy2DAsync(ws->xstage.p, sizeof(double2) * nin, xd, sizeof(double2) * ldx,
                             sizeof(double2) * nin, b, cudaMemcpyHostToDevice, s));
        if (usebeta)
            CK(cudaMemcpy2DAsync(ws->ystage.p, sizeof(double2) * nout, yd, sizeof(double2) * ldy,
                                 sizeof(double2) * nout, b, cudaMemcpyHostToDevice, s));
        xd = ws->xstage.p;
        yd = ws->ystage.p;
        lx = nin;
        ly = nout;
    }
    if (c->dir) {
        const DirProduct &pr = c->dir->prod[mode == 0 ? 0 : 1];
        const size_t need = size_t(pr.nin + pr.cin + pr.cout) * vector_slots(b) * (tangent ? 2 : 1);
        if (ws->arena.n < need) {
            drop_graphs(ws);
            ws->arena.alloc(need);
        }
    }
    if (tangent && ws->dxhat.n < ws->xhat.n) {
        ws->dxhat.alloc(ws->xhat.n);
        ws->dyhat.alloc(ws->xhat.n);
    }
    const ProductBuffers buf{ws->xt.p, ws->xhat.p, ws->yhat.p, ws->error.p, ws->far, ws->near};
    ProductLaunches count;
    // graph replay of repeated products on device arrays
    const bool graphable = ws->use_graphs && memspace == 1 && !tangent;
    const nca_workspace::GraphKey key{mode,    precision, b,   int(ws->far), int(ws->near), int(ws->profiling),
                                      int(ws->use_overlap),         x,   y,            ldx,           ldy,
                                      alpha.x, alpha.y,   beta.x, beta.y,     ws->gen};
    nca_workspace::Graph *graph = nullptr;
    bool capture = false;
    if (graphable) {
        for (auto &gr : ws->graphs)
            if (gr.key == key) graph = &gr;
        if (!graph)
            for (const auto &k : ws->seen)
                if (k == key) capture = true;
    }
    auto enqueue = [&]() -> int {
        if (c->dir && tangent) {
            if (int st = enqueue_dir_tangent(c, xd, lx, yd, ly, b, alpha, beta, ws->arena.p, ws->error.p, s, count))
                return st;
        } else if (c->dir) {
            ws->dir_stage.clear();
            DirTimer timer{&ws->dir_ev, &ws->dir_stage};
            if (int st = enqueue_dir_product(c, mode, precision, xd, lx, yd, ly, b, alpha, beta, ws->arena.p,
                                             ws->error.p, s, count, ws->profiling ? &timer : nullptr))
                return st;
        } else if (tangent) {
            if (int st = enqueue_tangent(c, xd, lx, yd, ly, b, alpha, beta, buf, ws->dxhat.p, ws->dyhat.p, s, count))
                return st;
        } else {
            ProductStreams ps;
            ps.aux = ws->use_overlap ? ws->aux : nullptr;
            ps.fork = ws->fork;
            ps.join = ws->join;
            ps.priority = ws->aux_priority;
            if (int st = enqueue_product(c, mode, precision, xd, lx, yd, ly, b, alpha, beta, buf, s,
                                         ws->profiling ? ws->stage_ev : nullptr, count, ps))
                return st;
        }
        return NCA_OK;
    };
    if (graph) {
        CK(cudaGraphLaunch(graph->exec, s));
        count.total = graph->launches;
        std::copy(graph->stage, graph->stage + kStages, count.stage);
    } else if (capture) {
        // a failed capture (an error return or a thrown CUDA error) is ended and discarded
        struct CaptureGuard {
            cudaStream_t s;
            bool active = true;
            ~CaptureGuard() {
                if (!active) return;
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(s, &g);
                if (g) cudaGraphDestroy(g);
            }
        } guard{s};
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        if (int st = enqueue()) return st;
        cudaGraph_t g = nullptr;
        guard.active = false;
        CK(cudaStreamEndCapture(s, &g));
        cudaGraphExec_t exec = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        CK(ie);
        if (ws->graphs.size() >= kGraphs) {
            cudaGraphExecDestroy(ws->graphs.front().exec);
            ws->graphs.erase(ws->graphs.begin());
        }
        nca_workspace::Graph gr;
        gr.key = key;
        gr.exec = exec;
        gr.launches = count.total;
        std::copy(count.stage, count.stage + kStages, gr.stage);
        ws->graphs.push_back(gr);
        CK(cudaGraphLaunch(exec, s));
    } else {
        if (int st = enqueue()) return st;
        if (graphable) {
            if (ws->seen.size() >= kGraphs) ws->seen.erase(ws->seen.begin());
            ws->seen.push_back(key);
        }
    }
    CK(cudaMemcpyAsync(ws->error_host, ws->error.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    if (memspace == 0)
        CK(cudaMemcpy2DAsync(y, sizeof(double2) * ldy, ws->ystage.p, sizeof(double2) * nout,
                             sizeof(double2) * nout, b, cudaMemcpyDeviceToHost, s));
    CK(cudaEventRecord(ws->e1, s));
    CK(cudaEventSynchronize(ws->e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ws->e0, ws->e1));
    ws->last_seconds = ms * 1e-3;
    ws->last_launches = count.total;
    if (ws->profiling && c->dir && !tangent) {
        // directional: the stages' event pairs summed per stage (no near-field stage of its own)
        for (int k = 0; k < kStages; ++k) {
            ws->stage_seconds[k] = 0.0;
            ws->stage_launches[k] = count.stage[k];
        }
        for (size_t i = 0; i < ws->dir_stage.size(); ++i) {
            float t = 0.f;
            CK(cudaEventElapsedTime(&t, ws->dir_ev[2 * i], ws->dir_ev[2 * i + 1]));
            ws->stage_seconds[ws->dir_stage[i]] += t * 1e-3;
        }
    } else if (ws->profiling && !tangent) {
        // gather, up, couple, down, near field, leaves (the sweeps and the near field overlap
        // when the workspace has its sweep stream)
        static const int from[kStages] = {EV_START, EV_GATHER, EV_UP, EV_COUPLE, EV_NEAR0, EV_LEAVES0};
        static const int to[kStages] = {EV_GATHER, EV_UP, EV_COUPLE, EV_DOWN, EV_NEAR1, EV_END};
        for (int k = 0; k < kStages; ++k) {
            float t = 0.f;
            CK(cudaEventElapsedTime(&t, ws->stage_ev[from[k]], ws->stage_ev[to[k]]));
            ws->stage_seconds[k] = t * 1e-3;
            ws->stage_launches[k] = count.stage[k];
        }
    }
    if (*ws->error_host == 2) return fail(NCA_ERR_TIMEOUT, "a bounded wait in the product kernel gave up");
    if (*ws->error_host != 0) return fail(NCA_ERR_CUDA, "internal: a product copy was misaligned and skipped");
    return NCA_OK;
}

// ---- batches: one block-diagonal core from several built cores ------------------------------
// Many independent problems of uneven size are applied as one operator: the batch renumbers the
// members' nodes, points, pairs and store offsets into one forest and copies the stores back to
// back, so every product stage (one launch per level of the deepest member, one coupling and one
// leaf launch) covers all members at once. x and y are the members' vectors stacked in order.


// dst = concatenation of counts[i] elements of parts[i]; with release, each part is freed once
// its copy has completed (moving the members' stores keeps the peak near one copy)
template <typename T>
void concat_device(DBuf<T> &dst, const std::vector<DBuf<T> *> &parts, const std::vector<size_t> &counts,
                   cudaStream_t s, bool release = false) {
    size_t total = 0;
    for (size_t c : counts) total += c;
    dst.alloc(total);
    size_t off = 0;
    for (size_t i = 0; i < parts.size(); ++i) {
        if (counts[i]) CK(cudaMemcpyAsync(dst.p + off, parts[i]->p, sizeof(T) * counts[i], cudaMemcpyDeviceToDevice, s));
        off += counts[i];
        if (release) {
            CK(cudaStreamSynchronize(s));
            parts[i]->release();
        }
    }
}

// appends v[0..n) + add to out (entries < 0 kept: "no node")
template <typename T, typename U>
void append_offset(std::vector<T> &out, const std::vector<U> &v, size_t n, int64_t add, bool keep_negative = false) {
    for (size_t i = 0; i < n; ++i) out.push_back(T(keep_negative && v[i] < 0 ? v[i] : v[i] + add));
}

// CSR pointer arrays: ptr of each member without its last entry, shifted; final total at the end
template <typename T>
void append_ptr(std::vector<T> &out, const std::vector<T> &ptr, int64_t add) {
    for (size_t i = 0; i + 1 < ptr.size(); ++i) out.push_back(T(ptr[i] + add));
}

void merge_trees(const std::vector<nca_core *> &cs, int sd, nca::Tree &T) {
    T = nca::Tree{};
    int64_t poff = 0;
    int noff = 0;
    for (const nca_core *c : cs) {
        const nca::Tree &M = c->tree[sd];
        append_offset(T.perm, M.perm, M.perm.size(), poff);
        append_offset(T.iperm, M.iperm, M.iperm.size(), poff);
        append_offset(T.begin, M.begin, M.begin.size(), poff);
        append_offset(T.end, M.end, M.end.size(), poff);
        append_offset(T.parent, M.parent, M.parent.size(), noff, true);
        append_offset(T.firstchild, M.firstchild, M.firstchild.size(), noff, true);
        T.nchildren.insert(T.nchildren.end(), M.nchildren.begin(), M.nchildren.end());
        T.level.insert(T.level.end(), M.level.begin(), M.level.end());
        T.center.insert(T.center.end(), M.center.begin(), M.center.end());
        T.radius.insert(T.radius.end(), M.radius.begin(), M.radius.end());
        T.nlevels = std::max(T.nlevels, M.nlevels);
        poff += M.npoints;
        noff += M.nnodes;
    }
    T.npoints = poff;
    T.nnodes = noff;
    T.levelptr.clear();  // members' nodes are not level-contiguous in a forest
}

void merge_core(const std::vector<nca_core *> &cs, nca_core *m, bool move, cudaStream_t s) {
    const size_t n = cs.size();
    m->device = cs[0]->device;
    m->maxrank = 0;
    m->f32 = true;
    for (const nca_core *c : cs) {
        m->maxrank = std::max(m->maxrank, c->maxrank);
        m->f32 = m->f32 && c->f32;
    }
    m->K = cs[0]->K;
    m->K.mat = nullptr;
    std::vector<int> noff[2], poff[2];
    for (int sd = 0; sd < 2; ++sd) {
        merge_trees(cs, sd, m->tree[sd]);
        int no = 0, po = 0;
        for (const nca_core *c : cs) {
            noff[sd].push_back(no);
            poff[sd].push_back(po);
            no += c->tree[sd].nnodes;
            po += int(c->tree[sd].npoints);
        }
    }
    // partition (test-node CSR and trial-node transposes)
    nca::Partition &P = m->part;
    int64_t nearoff = 0, faroff = 0, tnearoff = 0, tfaroff = 0;
    for (size_t i = 0; i < n; ++i) {
        const nca::Partition &Q = cs[i]->part;
        append_ptr(P.nearptr, Q.nearptr, nearoff);
        append_ptr(P.farptr, Q.farptr, faroff);
        append_ptr(P.tnearptr, Q.tnearptr, tnearoff);
        append_ptr(P.tfarptr, Q.tfarptr, tfaroff);
        append_offset(P.nearnodes, Q.nearnodes, Q.nearnodes.size(), noff[1][i]);
        append_offset(P.farnodes, Q.farnodes, Q.farnodes.size(), noff[1][i]);
        append_offset(P.tnearnodes, Q.tnearnodes, Q.tnearnodes.size(), noff[0][i]);
        append_offset(P.tfarnodes, Q.tfarnodes, Q.tfarnodes.size(), noff[0][i]);
        nearoff += Q.nearnodes.size();
        faroff += Q.farnodes.size();
        tnearoff += Q.tnearnodes.size();
        tfaroff += Q.tfarnodes.size();
    }
    P.nearptr.push_back(int32_t(nearoff));
    P.farptr.push_back(int32_t(faroff));
    P.tnearptr.push_back(int32_t(tnearoff));
    P.tfarptr.push_back(int32_t(tfaroff));
    // sides: node arrays, bases, plans
    for (int sd = 0; sd < 2; ++sd) {
        DevSide &d = m->side[sd];
        const nca::Tree &T = m->tree[sd];
        d.nnodes = T.nnodes;
        d.nlevels = T.nlevels;
        d.npts = T.npoints;
        d.perm.upload(T.perm, s);
        d.begin.upload(T.begin, s);
        d.end.upload(T.end, s);
        d.firstchild.upload(T.firstchild, s);
        d.nchildren.upload(T.nchildren, s);
        std::vector<DBuf<double> *> pts;
        std::vector<size_t> npts;
        for (nca_core *c : cs) {
            pts.push_back(&c->side[sd].pts);
            npts.push_back(size_t(3 * c->side[sd].npts));
        }
        concat_device(d.pts, pts, npts, s, move);
        d.h_rank.clear();
        d.h_nrows.clear();
        d.h_fpptr.clear();
        d.h_fpidx.clear();
        d.h_xoff.clear();
        d.h_cptr.clear();
        d.h_piv.assign(size_t(T.nnodes) * m->maxrank, 0);
        int64_t xo = 0, co = 0, fo = 0;
        std::vector<DBuf<double2> *> X, XT;
        std::vector<DBuf<float2> *> X32, XT32;
        std::vector<size_t> xn;
        for (size_t i = 0; i < n; ++i) {
            DevSide &e = cs[i]->side[sd];
            const int nn = e.nnodes;
            d.h_rank.insert(d.h_rank.end(), e.h_rank.begin(), e.h_rank.end());
            d.h_nrows.insert(d.h_nrows.end(), e.h_nrows.begin(), e.h_nrows.end());
            append_ptr(d.h_fpptr, e.h_fpptr, fo);
            append_offset(d.h_fpidx, e.h_fpidx, e.h_fpidx.size(), poff[sd][i]);
            append_ptr(d.h_xoff, e.h_xoff, xo);
            append_ptr(d.h_cptr, e.h_cptr, co);
            for (int t = 0; t < nn; ++t)
                for (int r = 0; r < e.h_rank[t]; ++r)
                    d.h_piv[size_t(noff[sd][i] + t) * m->maxrank + r] =
                        e.h_piv[size_t(t) * cs[i]->maxrank + r] + poff[sd][i];
            fo += e.h_fpptr.back();
            xo += e.h_xoff.back();
            co += e.h_cptr.back();
            X.push_back(&e.X);
            XT.push_back(&e.XT);
            X32.push_back(&e.X32);
            XT32.push_back(&e.XT32);
            xn.push_back(size_t(e.h_xoff.back()));
        }
        d.h_fpptr.push_back(int32_t(fo));
        d.h_xoff.push_back(xo);
        d.h_cptr.push_back(co);
        d.rank.upload(d.h_rank, s);
        d.nrows.upload(d.h_nrows, s);
        d.xoff.upload(d.h_xoff, s);
        d.cptr.upload(d.h_cptr, s);
        concat_device(d.X, X, xn, s, move);
        concat_device(d.XT, XT, xn, s, move);
        if (m->f32) {
            concat_device(d.X32, X32, xn, s, move);
            concat_device(d.XT32, XT32, xn, s, move);
        }
        // level lists by depth: up deepest first, down root first, over all members
        d.up.ptr.assign(1, 0);
        d.up.nodes.clear();
        d.up.mcap.clear();
        d.down.ptr.assign(1, 0);
        d.down.nodes.clear();
        d.down.mcap.clear();
        for (int pass = 0; pass < 2; ++pass) {
            LevelLists &L = pass == 0 ? d.up : d.down;
            for (int g = 0; g < T.nlevels; ++g) {
                const int depth = pass == 0 ? T.nlevels - 1 - g : g;
                int mc = 0;
                for (size_t i = 0; i < n; ++i) {
                    const DevSide &e = cs[i]->side[sd];
                    const LevelLists &Le = pass == 0 ? e.up : e.down;
                    const int ge = pass == 0 ? e.nlevels - 1 - depth : depth;  // member's group
                    if (ge < 0 || ge + 1 >= int(Le.ptr.size())) continue;
                    for (int k = Le.ptr[ge]; k < Le.ptr[ge + 1]; ++k) L.nodes.push_back(Le.nodes[k] + noff[sd][i]);
                    mc = std::max(mc, Le.mcap[ge]);
                }
                L.ptr.push_back(int32_t(L.nodes.size()));
                L.mcap.push_back(mc);
            }
            L.d_nodes.upload(L.nodes, s);
        }
        std::vector<int32_t> leaves;
        d.leafcap = 0;
        for (int node = 0; node < T.nnodes; ++node)
            if (T.isleaf(node)) {
                leaves.push_back(node);
                d.leafcap = std::max(d.leafcap, T.size(node));
            }
        d.nleaves = int(leaves.size());
        d.leaves.upload(leaves, s);
    }
    // couplings: test-CSR blocks (cfoff) and their trial-CSR transposes (ctoff)
    {
        std::vector<int64_t> ctoff;
        std::vector<DBuf<double2> *> Cp, CTp;
        std::vector<DBuf<float2> *> C32p, CT32p;
        std::vector<size_t> cn, ctn;
        int64_t co = 0, cto = 0;
        m->h_cfoff.clear();
        for (size_t i = 0; i < n; ++i) {
            nca_core *c = cs[i];
            const size_t npair = c->part.farnodes.size(), ntp = c->part.tfarnodes.size();
            append_ptr(m->h_cfoff, c->h_cfoff, co);
            const std::vector<int64_t> h_ctoff = download_now(c->ctoff, ntp + 1);
            append_ptr(ctoff, h_ctoff, cto);
            co += c->h_cfoff[npair];
            cto += h_ctoff[ntp];
            Cp.push_back(&c->C);
            CTp.push_back(&c->CT);
            C32p.push_back(&c->C32);
            CT32p.push_back(&c->CT32);
            cn.push_back(size_t(c->h_cfoff[npair]));
            ctn.push_back(size_t(h_ctoff[ntp]));
        }
        m->h_cfoff.push_back(co);
        ctoff.push_back(cto);
        m->cfoff.upload(m->h_cfoff, s);
        m->ctoff.upload(ctoff, s);
        concat_device(m->C, Cp, cn, s, move);
        concat_device(m->CT, CTp, ctn, s, move);
        if (m->f32) {
            concat_device(m->C32, C32p, cn, s, move);
            concat_device(m->CT32, CT32p, ctn, s, move);
        }
        m->farptr.upload(P.farptr, s);
        m->farnodes.upload(P.farnodes, s);
        m->tfarptr.upload(P.tfarptr, s);
        m->tfarnodes.upload(P.tfarnodes, s);
        // coupling output nodes of all members, largest work first
        const std::vector<int32_t> &rt = m->side[0].h_rank, &rs = m->side[1].h_rank;
        std::vector<int32_t> fwd, rev;
        std::vector<int64_t> wf(rt.size(), 0), wr(rs.size(), 0);
        for (size_t t = 0; t < rt.size(); ++t) {
            if (rt[t] <= 0) continue;
            fwd.push_back(int32_t(t));
            for (int k = P.farptr[t]; k < P.farptr[t + 1]; ++k) wf[t] += int64_t(rt[t]) * rs[P.farnodes[k]];
        }
        for (size_t u = 0; u < rs.size(); ++u) {
            if (rs[u] <= 0) continue;
            rev.push_back(int32_t(u));
            for (int k = P.tfarptr[u]; k < P.tfarptr[u + 1]; ++k) wr[u] += int64_t(rs[u]) * rt[P.tfarnodes[k]];
        }
        std::stable_sort(fwd.begin(), fwd.end(), [&](int a, int b) { return wf[a] > wf[b]; });
        std::stable_sort(rev.begin(), rev.end(), [&](int a, int b) { return wr[a] > wr[b]; });
        m->n_couple_fwd = int(fwd.size());
        m->n_couple_rev = int(rev.size());
        m->couple_fwd.upload(fwd, s);
        m->couple_rev.upload(rev, s);
    }
    // near field
    {
        std::vector<int64_t> ntoff;
        std::vector<DBuf<double2> *> Np, NTp;
        std::vector<DBuf<float2> *> N32p, NT32p;
        std::vector<size_t> nn, ntn;
        int64_t no = 0, nto = 0, ro = 0;
        m->h_nfoff.clear();
        m->h_noff.clear();
        m->h_ncols.clear();
        for (size_t i = 0; i < n; ++i) {
            nca_core *c = cs[i];
            const size_t npair = c->part.nearnodes.size(), ntp = c->part.tnearnodes.size();
            append_ptr(m->h_nfoff, c->h_nfoff, no);
            append_ptr(m->h_noff, c->h_noff, ro);
            m->h_ncols.insert(m->h_ncols.end(), c->h_ncols.begin(), c->h_ncols.end());
            const std::vector<int64_t> h_ntoff = download_now(c->ntoff, ntp + 1);
            append_ptr(ntoff, h_ntoff, nto);
            no += c->h_nfoff[npair];
            nto += h_ntoff[ntp];
            ro += c->h_noff.back();
            Np.push_back(&c->N);
            NTp.push_back(&c->NT);
            N32p.push_back(&c->N32);
            NT32p.push_back(&c->NT32);
            nn.push_back(size_t(c->h_nfoff[npair]));
            ntn.push_back(size_t(h_ntoff[ntp]));
        }
        m->h_nfoff.push_back(no);
        m->h_noff.push_back(ro);
        ntoff.push_back(nto);
        m->nfoff.upload(m->h_nfoff, s);
        m->ntoff.upload(ntoff, s);
        concat_device(m->N, Np, nn, s, move);
        concat_device(m->NT, NTp, ntn, s, move);
        if (m->f32) {
            concat_device(m->N32, N32p, nn, s, move);
            concat_device(m->NT32, NT32p, ntn, s, move);
        }
        m->nearptr.upload(P.nearptr, s);
        m->nearnodes.upload(P.nearnodes, s);
        m->tnearptr.upload(P.tnearptr, s);
        m->tnearnodes.upload(P.tnearnodes, s);
    }
    m->batch = true;
    if (move)
        for (nca_core *c : cs) c->moved = true;
    // storage summary: sums of the members'
    nca_core_info &I = m->info;
    I = nca_core_info{};
    for (const nca_core *c : cs) {
        const nca_core_info &J = c->info;
        I.ntest += J.ntest;
        I.ntrial += J.ntrial;
        I.nnodes_test += J.nnodes_test;
        I.nnodes_trial += J.nnodes_trial;
        I.ncoeff_test += J.ncoeff_test;
        I.ncoeff_trial += J.ncoeff_trial;
        I.near_entries += J.near_entries;
        I.coupling_entries += J.coupling_entries;
        I.basis_entries_test += J.basis_entries_test;
        I.basis_entries_trial += J.basis_entries_trial;
        I.transfer_entries_test += J.transfer_entries_test;
        I.transfer_entries_trial += J.transfer_entries_trial;
        I.nfarpairs += J.nfarpairs;
        I.nnearpairs += J.nnearpairs;
        I.build_seconds += J.build_seconds;
        I.build_seconds_host += J.build_seconds_host;
    }
}

// ---- allocation-free product ------------------------------------------------------------
// Callers that cannot allocate device memory: a host whose own pool (Julia's CUDA.jl, PyTorch's
// caching allocator) has reserved nearly all of HBM, so a cudaMalloc inside the library fails or
// fragments the pool, and callers on a path that must not synchronise on cudaMalloc/cudaFree.
// nca_apply_static keeps every intermediate buffer of the product (gathered input, xhat, yhat,
// error word) in this file-scope array instead: NCA_STATIC_SCRATCH_BYTES per device, reserved by
// the CUDA runtime when it loads the library's module on that device (at the library load under
// CUDA_MODULE_LOADING=EAGER, else at the first use on the device, which for a caller of this entry
// point alone is its first call there) and held until the process exits; the call itself never
// allocates.
static __device__ __align__(256) unsigned char g_static_scratch[NCA_STATIC_SCRATCH_BYTES];

constexpr int kMaxStaticDevices = 64;
std::mutex g_static_setup;
void *g_static_base[kMaxStaticDevices] = {};
std::atomic<bool> g_static_busy[kMaxStaticDevices];

inline size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

// Device address of this device's scratch array; the first call per device looks it up (with
// that device current), which loads the module holding the array.
int static_scratch_base(int device, unsigned char **base) {
    std::lock_guard<std::mutex> lock(g_static_setup);
    if (!g_static_base[device]) {
        void *p = nullptr;
        const cudaError_t rc = cudaGetSymbolAddress(&p, g_static_scratch);
        if (rc != cudaSuccess)
            return fail(NCA_ERR_CUDA, std::string("cudaGetSymbolAddress(static product scratch): ") +
                                          cudaGetErrorString(rc));
        g_static_base[device] = p;
    }
    *base = static_cast<unsigned char *>(g_static_base[device]);
    return NCA_OK;
}

int apply_static_impl(nca_core *c, int mode, int precision, const void *x, int64_t ldx, void *y, int64_t ldy,
                      int64_t nrhs, double2 alpha, double2 beta, cudaStream_t s) {
    if (c->moved) return fail(NCA_ERR_ARG, "the core's stores were moved into a batch");
    if (c->dir) return fail(NCA_ERR_ARG, "nca_apply_static does not take directional cores; use nca_apply");
    if (int st = check_product_args(c, mode, precision, ldx, ldy, nrhs)) return st;
    if (nrhs == 0) return NCA_OK;
    if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15)
        return fail(NCA_ERR_ARG, "x and y must be 16-byte aligned device arrays");
    const int in = mode == 0 ? 1 : 0, out = 1 - in;
    const int b = int(std::min<int64_t>(nrhs, 1 << 30));
    const size_t vs = size_t(vector_stride(b));
    // layout: error word | xt (nin x vs) | xhat (input coefficients x vs) | yhat (output coefficients x vs)
    const size_t o_xt = 256;
    const size_t o_xhat = o_xt + align256(sizeof(double2) * size_t(c->side[in].npts) * vs);
    const size_t o_yhat = o_xhat + align256(sizeof(double2) * size_t(c->side[in].h_cptr.back()) * vs);
    const size_t need = o_yhat + align256(sizeof(double2) * size_t(c->side[out].h_cptr.back()) * vs);
    if (nrhs != b || need > size_t(NCA_STATIC_SCRATCH_BYTES))
        return fail(NCA_ERR_ARG, "nca_apply_static: " + std::to_string(nrhs) + " right-hand sides need " +
                                     std::to_string(need) + " bytes of scratch, more than the fixed " +
                                     std::to_string(size_t(NCA_STATIC_SCRATCH_BYTES)) +
                                     " (NCA_STATIC_SCRATCH_BYTES); use nca_apply or fewer right-hand sides");
    if (c->device < 0 || c->device >= kMaxStaticDevices)
        return fail(NCA_ERR_ARG, "nca_apply_static supports devices 0..63");
    CK(cudaSetDevice(c->device));
    // the call reads its status back and waits for its stream, which a stream capture forbids
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(s, &cap));
    if (cap != cudaStreamCaptureStatusNone)
        return fail(NCA_ERR_ARG, "nca_apply_static cannot be captured in a CUDA graph (it waits for its stream)");
    unsigned char *base = nullptr;
    if (int st = static_scratch_base(c->device, &base)) return st;
    bool expected = false;
    if (!g_static_busy[c->device].compare_exchange_strong(expected, true))
        return fail(NCA_ERR_BUSY, "nca_apply_static: another call on this device is using the static scratch");
    // the flag is released only once no kernel of this call can touch the scratch any more: after
    // a failure past the first launch the stream is drained first (its status ignored)
    struct Release {
        std::atomic<bool> &flag;
        cudaStream_t s;
        bool launched = false;
        ~Release() {
            if (launched) cudaStreamSynchronize(s);
            flag.store(false);
        }
    } release{g_static_busy[c->device], s};
    const ProductBuffers buf{reinterpret_cast<double2 *>(base + o_xt), reinterpret_cast<double2 *>(base + o_xhat),
                             reinterpret_cast<double2 *>(base + o_yhat), reinterpret_cast<int32_t *>(base), true,
                             true};
    // Only the error word must start at zero: every xt row is gathered, every xhat / yhat block
    // is written (up sweep, coupling) before it is read.
    release.launched = true;
    CK(cudaMemsetAsync(buf.error, 0, sizeof(int32_t), s));
    ProductLaunches count;
    if (int st = enqueue_product(c, mode, precision, reinterpret_cast<const double2 *>(x), ldx,
                                 reinterpret_cast<double2 *>(y), ldy, b, alpha, beta, buf, s, nullptr, count))
        return st;
    int32_t err = 0;
    CK(cudaMemcpyAsync(&err, buf.error, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (err == 2) return fail(NCA_ERR_TIMEOUT, "a bounded wait in the product kernel gave up");
    if (err != 0) return fail(NCA_ERR_CUDA, "internal: a product copy was misaligned and skipped");
    return NCA_OK;
}

int entries_impl(const nca_kernel_desc *kernel, const double *testpoints, int64_t ntest, const double *trialpoints,
                 int64_t ntrial, const int64_t *ii, const int64_t *jj, int64_t n, int32_t device, double *out,
                 int deriv);

}  // namespace

// ---- directional cores on a frozen skeleton: refills and d/dk stores -------------------------
// X of every item of one side at kernel K (mode 0: K[rows, sigma] K[tau, sigma]^-1) or its
// wavenumber derivative (mode 1, from Xin = X at K), at the build's offsets.
void fill_dir_bases(nca_core *c, int sd, int mode, const KernelParams &K, const KernelParams &dK, const double2 *Xin,
                    double2 *Xout, cudaStream_t s) {
    DirItems &d = c->dir->side[sd];
    std::vector<int32_t> items;
    int mcap = 1, rcap = 1;
    for (int it = 0; it < d.nitems; ++it)
        if (d.h_rank[it] > 0) {
            items.push_back(it);
            mcap = std::max(mcap, d.h_nrows[it]);
            rcap = std::max(rcap, d.h_rank[it]);
        }
    if (items.empty()) return;
    const size_t sm = values_smem_bytes(mcap, rcap, mode);
    if (sm > size_t(kMaxSmem))
        throw Failure(NCA_ERR_ARG, "a cross block of the frozen skeleton does not fit in shared memory");
    CK(cudaFuncSetAttribute(k_level_values, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    DBuf<int32_t> status, ditems;
    status.alloc(4);
    status.zero(s);
    ditems.upload(items, s);
    const DevSide &ds = c->side[sd];
    ValueArgs a{};
    a.K = K;
    a.dK = dK;
    a.side = sd;
    a.mode = mode;
    a.own_pts = ds.pts.p;
    a.far_pts = c->side[1 - sd].pts.p;
    a.perm = ds.perm.p;
    a.begin = ds.begin.p;
    a.end = ds.end.p;
    a.firstchild = ds.firstchild.p;
    a.nchildren = ds.nchildren.p;
    a.rank = d.rank.p;
    a.piv = d.piv.p;
    a.cpiv = d.cpiv.p;
    a.item_node = d.item_node.p;
    a.item_basis = d.item_basis.p;
    a.item_chptr = d.item_chptr.p;
    a.item_chidx = d.item_chidx.p;
    a.maxrank = c->maxrank;
    a.Xin = Xin;
    a.Xout = Xout;
    a.xoff = d.xoff.p;
    a.status = status.p;
    k_level_values<<<int(items.size()), 256, sm, s>>>(a, ditems.p, mcap, rcap);
    CK(cudaGetLastError());
    const std::vector<int32_t> st = status.download(s);
    if (st[0] == 1) {
        set_singular(sd, st[1], st[2], st[3]);
        throw Failure(NCA_ERR_SINGULAR, "SingularCrossMatrixError: the frozen cross matrix of " +
                                            std::string(sd == 0 ? "test" : "trial") + " item " +
                                            std::to_string(st[1]) + " is singular at this wavenumber");
    }
    if (st[0] == 2) throw Failure(NCA_ERR_CUDA, "internal: a frozen cross block exceeds its planned capacity");
}

// Every stage store of both orientations from the sides' operators X (and their transposes XT),
// the couplings and the near field at K: the value stores (deriv = false) or the d/dk stores.
void fill_dir_stores(nca_core *c, const KernelParams &K, double2 *const X[2], double2 *const XT[2], bool deriv,
                     cudaStream_t s) {
    DirCore &D = *c->dir;
    for (int m = 0; m < 2; ++m) {
        const int I = m == 0 ? 1 : 0, O = 1 - I;
        DirProduct &pr = D.prod[m];
        auto copy = [&](GatherStage &G, const double2 *src) {
            DBuf<double2> &dst = deriv ? G.dM : G.M;
            if (deriv && dst.n != G.M.n) dst.alloc(G.M.n);
            if (G.ncopies)
                launch_copy_blocks<double2>(src, G.c_soff.p, G.c_ld.p, G.c_rows.p, G.c_cols.p, G.c_doff.p, G.ncopies,
                                            dst.p, s);
            CK(cudaGetLastError());
        };
        if (pr.same) continue;  // its stages are the forward product's, refilled above
        copy(pr.up, XT[I]);
        copy(pr.down, X[O]);
        copy(pr.leaves, X[O]);
    }
    GatherStage &CN = D.prod[0].couple, &CTs = D.prod[1].couple;
    DBuf<double2> &C = deriv ? CN.dM : CN.M, &CT = deriv ? CTs.dM : CTs.M;
    if (deriv) {
        C.alloc(CN.M.n);
        CT.alloc(CTs.M.n);
    }
    CouplingArgs a{};
    a.K = K;
    a.test_pts = c->side[0].pts.p;
    a.trial_pts = c->side[1].pts.p;
    a.pair_t = D.cpair_it.p;
    a.pair_s = D.cpair_is.p;
    a.rank_t = D.side[0].rank.p;
    a.rank_s = D.side[1].rank.p;
    a.piv_t = D.side[0].piv.p;
    a.piv_s = D.side[1].piv.p;
    a.maxrank = c->maxrank;
    a.coff = D.ccoff.p;
    a.npairs = D.npairs;
    a.C = C.p;
    if (D.npairs > 0) {
        k_couplings<<<launch_grid(D.npairs, 16), 256, 0, s>>>(a);
        CK(cudaGetLastError());
    }
    launch_transpose_blocks<double2>(C.p, D.ctr_in.p, D.ctr_rows.p, D.ctr_cols.p, D.ctr_off.p, D.ntr, CT.p, s);
    CK(cudaGetLastError());
    if (deriv) {
        c->dN.alloc(c->N.n);
        c->dNT.alloc(c->NT.n);
    }
    fill_near(c, K, deriv ? c->dN.p : c->N.p, deriv ? c->dNT.p : c->NT.p, s);
}

// complex-FP32 copies of a directional core's stage stores and near field
void make_dir_f32(nca_core *c, cudaStream_t s) {
    auto down = [&](DBuf<double2> &src, DBuf<float2> &dst) {
        if (dst.n != src.n) dst.alloc(src.n);
        if (src.n) k_to_f32<<<launch_grid(int64_t(src.n) / 256 + 1, 8), 256, 0, s>>>(src.p, dst.p, int64_t(src.n));
        CK(cudaGetLastError());
    };
    for (DirProduct &pr : c->dir->prod)
        for (GatherStage *G : pr.own_stages()) down(G->M, G->M32);
    down(c->N, c->N32);
    down(c->NT, c->NT32);
}

// drops the d/dk stores of a directional core (they belong to the wavenumber they were prepared at)
void drop_dir_dk(nca_core *c) {
    c->dN.release();
    c->dNT.release();
    for (DirProduct &pr : c->dir->prod)
        for (GatherStage *G : pr.own_stages()) G->dM.release();
    c->has_dk = false;
}

void set_dir_wavenumber(nca_core *c, double k, cudaStream_t s) {
    KernelParams K = c->K;
    K.k = k;
    K.deriv = 0;
    // new operators first (a singular frozen cross matrix leaves the core unchanged)
    DBuf<double2> X[2], XT[2];
    for (int sd = 0; sd < 2; ++sd) {
        DirItems &d = c->dir->side[sd];
        X[sd].alloc(d.X.n);
        XT[sd].alloc(d.X.n);
        fill_dir_bases(c, sd, 0, K, K, nullptr, X[sd].p, s);
        launch_transpose_blocks<double2>(X[sd].p, d.xoff.p, d.nrows.p, d.rank.p, d.xoff.p, d.nitems, XT[sd].p, s);
        CK(cudaGetLastError());
    }
    double2 *const xs[2] = {X[0].p, X[1].p}, *const xts[2] = {XT[0].p, XT[1].p};
    fill_dir_stores(c, K, xs, xts, false, s);
    for (int sd = 0; sd < 2; ++sd) std::swap(c->dir->side[sd].X.p, X[sd].p);
    c->K.k = k;
    if (c->f32) make_dir_f32(c, s);
    drop_dir_dk(c);
    CK(cudaStreamSynchronize(s));
}

void prepare_dir_dk(nca_core *c, cudaStream_t s) {
    KernelParams dK = c->K;
    dK.deriv = 1;
    DBuf<double2> dX[2], dXT[2];
    for (int sd = 0; sd < 2; ++sd) {
        DirItems &d = c->dir->side[sd];
        dX[sd].alloc(d.X.n);
        dXT[sd].alloc(d.X.n);
        fill_dir_bases(c, sd, 1, c->K, dK, d.X.p, dX[sd].p, s);
        launch_transpose_blocks<double2>(dX[sd].p, d.xoff.p, d.nrows.p, d.rank.p, d.xoff.p, d.nitems, dXT[sd].p, s);
        CK(cudaGetLastError());
    }
    double2 *const xs[2] = {dX[0].p, dX[1].p}, *const xts[2] = {dXT[0].p, dXT[1].p};
    fill_dir_stores(c, dK, xs, xts, true, s);
    CK(cudaStreamSynchronize(s));
    c->has_dk = true;
}

// ---- serialised cores ---------------------------------------------------------------------
// File layout (little-endian, native sizes): an 8-byte tag, the format number, the core's options
// and kernel, the points, both trees, the partition, then per side the skeleton (SavedSide); every
// array is its element count (int64) followed by its elements.
constexpr char kCoreTag[8] = {'N', 'C', 'A', 'B', '2', '0', '0', 'C'};
constexpr uint32_t kCoreFormat = 1;

struct FileOut {
    FILE *f = nullptr;
    ~FileOut() {
        if (f) std::fclose(f);
    }
    void raw(const void *p, size_t n) {
        if (n && std::fwrite(p, 1, n, f) != n) throw Failure(NCA_ERR_ARG, "nca_core_save: write failed");
    }
    template <typename T>
    void pod(const T &v) {
        raw(&v, sizeof(T));
    }
    template <typename T>
    void vec(const std::vector<T> &v) {
        pod<int64_t>(int64_t(v.size()));
        raw(v.data(), sizeof(T) * v.size());
    }
};

struct FileIn {
    FILE *f = nullptr;
    int64_t left = 0;  // bytes not yet read: bounds every array count
    ~FileIn() {
        if (f) std::fclose(f);
    }
    void raw(void *p, size_t n) {
        if (int64_t(n) > left || (n && std::fread(p, 1, n, f) != n))
            throw Failure(NCA_ERR_ARG, "nca_core_load: the file is truncated or not a saved core");
        left -= int64_t(n);
    }
    template <typename T>
    T pod() {
        T v{};
        raw(&v, sizeof(T));
        return v;
    }
    template <typename T>
    void vec(std::vector<T> &v) {
        const int64_t n = pod<int64_t>();
        if (n < 0 || n > left / int64_t(sizeof(T)))
            throw Failure(NCA_ERR_ARG, "nca_core_load: the file is truncated or not a saved core");
        v.resize(size_t(n));
        raw(v.data(), sizeof(T) * size_t(n));
    }
};

template <typename IO, typename TreeT>
void tree_io(IO &io, TreeT &T) {
    io.vec(T.perm);
    io.vec(T.iperm);
    io.vec(T.begin);
    io.vec(T.end);
    io.vec(T.parent);
    io.vec(T.firstchild);
    io.vec(T.nchildren);
    io.vec(T.level);
    io.vec(T.center);
    io.vec(T.radius);
    io.vec(T.levelptr);
}

template <typename IO, typename PartT>
void partition_io(IO &io, PartT &P) {
    io.vec(P.nearptr);
    io.vec(P.nearnodes);
    io.vec(P.farptr);
    io.vec(P.farnodes);
    io.vec(P.tnearptr);
    io.vec(P.tnearnodes);
    io.vec(P.tfarptr);
    io.vec(P.tfarnodes);
}

template <typename IO, typename PlanT>
void plan_io(IO &io, PlanT &D) {
    io.vec(D.farptr);
    io.vec(D.farnodes);
    io.vec(D.dirptr);
    io.vec(D.dirs);
    io.vec(D.dirvec);
    io.vec(D.dirfarptr);
    io.vec(D.chdirptr);
    io.vec(D.chdirmap);
    io.vec(D.invptr);
    io.vec(D.invidx);
    io.vec(D.item_node);
    io.vec(D.item_basis);
    io.vec(D.item_chptr);
    io.vec(D.item_chidx);
}

template <typename IO, typename SideT>
void saved_side_io(IO &io, SideT &v, bool dir) {
    io.vec(v.rank);
    io.vec(v.nrows);
    io.vec(v.piv);
    io.vec(v.cpiv);
    io.vec(v.fpptr);
    io.vec(v.fpidx);
    io.vec(v.xoff);
    io.vec(v.X);
    if (dir) plan_io(io, v.plan);
}

// every array of a read tree / partition / skeleton has the size its counts imply
void check_loaded(const nca::Tree &T, const char *what) {
    const size_t n = size_t(T.nnodes);
    const bool ok = T.nnodes > 0 && T.nlevels > 0 && T.perm.size() == size_t(T.npoints) &&
                    T.iperm.size() == size_t(T.npoints) && T.begin.size() == n && T.end.size() == n &&
                    T.parent.size() == n && T.firstchild.size() == n && T.nchildren.size() == n &&
                    T.level.size() == n && T.center.size() == 3 * n && T.radius.size() == n &&
                    T.levelptr.size() == size_t(T.nlevels) + 1;
    if (!ok) throw Failure(NCA_ERR_ARG, std::string("nca_core_load: inconsistent ") + what);
}

void save_core(const nca_core *c, const char *path) {
    if (c->batch) throw Failure(NCA_ERR_ARG, "nca_core_save: a batch is not saved (save its members)");
    if (c->moved) throw Failure(NCA_ERR_ARG, "the core's stores were moved into a batch");
    CK(cudaSetDevice(c->device));
    cudaStream_t s = nullptr;
    FileOut out;
    out.f = std::fopen(path, "wb");
    if (!out.f) throw Failure(NCA_ERR_ARG, std::string("nca_core_save: cannot open ") + path);
    out.raw(kCoreTag, sizeof(kCoreTag));
    out.pod<uint32_t>(kCoreFormat);
    const bool dir = c->dir != nullptr;
    out.pod<int32_t>(dir);
    out.pod<int32_t>(c->f32);
    out.pod<int32_t>(c->maxrank);
    out.pod<int32_t>(c->K.kind);
    out.pod<int32_t>(c->K.sign);
    out.pod<double>(c->K.k);
    out.pod<double>(c->K.rmin);
    out.pod<int64_t>(c->K.ldmat);
    out.pod<double>(c->wb.k);
    out.pod<double>(c->wb.etalf);
    out.pod<double>(c->wb.etahf);
    out.pod<double>(c->wb.gamma);
    for (int sd = 0; sd < 2; ++sd) {
        out.pod<int64_t>(c->tree[sd].npoints);
        out.pod<int32_t>(c->tree[sd].nnodes);
        out.pod<int32_t>(c->tree[sd].nlevels);
    }
    for (int sd = 0; sd < 2; ++sd) out.vec(c->side[sd].pts.download(s));
    out.vec(c->K.kind == NCA_KERNEL_MATRIX ? c->kmat.download(s) : std::vector<double2>());
    for (int sd = 0; sd < 2; ++sd) tree_io(out, const_cast<nca::Tree &>(c->tree[sd]));
    partition_io(out, const_cast<nca::Partition &>(c->part));
    for (int sd = 0; sd < 2; ++sd) {
        SavedSide v;
        if (dir) {
            const DirItems &d = c->dir->side[sd];
            v.rank = d.h_rank;
            v.nrows = d.h_nrows;
            v.piv = d.piv.download(s);
            v.cpiv = d.cpiv.download(s);
            v.xoff = d.h_xoff;
            v.X = d.X.download(s);
            v.plan = d.plan;
        } else {
            const DevSide &d = c->side[sd];
            v.rank = d.h_rank;
            v.nrows = d.h_nrows;
            v.piv = d.h_piv;
            v.cpiv = d.cpiv.download(s);
            v.fpptr = d.h_fpptr;
            v.fpidx = d.h_fpidx;
            v.xoff = d.h_xoff;
            v.X = d.X.download(s);
        }
        saved_side_io(out, v, dir);
    }
    if (std::fflush(out.f) != 0) throw Failure(NCA_ERR_ARG, "nca_core_save: write failed");
}

nca_core *load_core(const char *path, int device) {
    FileIn in;
    in.f = std::fopen(path, "rb");
    if (!in.f) throw Failure(NCA_ERR_ARG, std::string("nca_core_load: cannot open ") + path);
    std::fseek(in.f, 0, SEEK_END);
    in.left = std::ftell(in.f);
    std::fseek(in.f, 0, SEEK_SET);
    char tag[8];
    in.raw(tag, sizeof(tag));
    if (std::memcmp(tag, kCoreTag, sizeof(tag)) != 0) throw Failure(NCA_ERR_ARG, "nca_core_load: not a saved core");
    if (in.pod<uint32_t>() != kCoreFormat) throw Failure(NCA_ERR_ARG, "nca_core_load: unknown format version");
    auto c = std::make_unique<nca_core>();
    const bool dir = in.pod<int32_t>() != 0;
    c->device = device;
    c->f32 = in.pod<int32_t>() != 0;
    c->maxrank = in.pod<int32_t>();
    nca_kernel_desc kd{};
    kd.kind = in.pod<int32_t>();
    kd.sign = in.pod<int32_t>();
    kd.k = in.pod<double>();
    kd.rmin = in.pod<double>();
    kd.ldmatrix = in.pod<int64_t>();
    c->wb.k = in.pod<double>();
    c->wb.etalf = in.pod<double>();
    c->wb.etahf = in.pod<double>();
    c->wb.gamma = in.pod<double>();
    for (int sd = 0; sd < 2; ++sd) {
        c->tree[sd].npoints = in.pod<int64_t>();
        c->tree[sd].nnodes = in.pod<int32_t>();
        c->tree[sd].nlevels = in.pod<int32_t>();
    }
    if (c->maxrank < 1 || c->maxrank > 128) throw Failure(NCA_ERR_ARG, "nca_core_load: bad maxrank");
    std::vector<double> pts[2];
    for (int sd = 0; sd < 2; ++sd) {
        in.vec(pts[sd]);
        if (pts[sd].size() != 3 * size_t(c->tree[sd].npoints))
            throw Failure(NCA_ERR_ARG, "nca_core_load: point count differs from the tree's");
    }
    std::vector<double2> mat;
    in.vec(mat);
    kd.matrix = reinterpret_cast<const double *>(mat.data());
    for (int sd = 0; sd < 2; ++sd) {
        tree_io(in, c->tree[sd]);
        check_loaded(c->tree[sd], sd == 0 ? "test tree" : "trial tree");
    }
    partition_io(in, c->part);
    if (c->part.nearptr.size() != size_t(c->tree[0].nnodes) + 1 ||
        c->part.tfarptr.size() != size_t(c->tree[1].nnodes) + 1)
        throw Failure(NCA_ERR_ARG, "nca_core_load: inconsistent partition");
    SavedCore sv;
    for (int sd = 0; sd < 2; ++sd) {
        saved_side_io(in, sv.side[sd], dir);
        const SavedSide &v = sv.side[sd];
        const size_t n = dir ? v.plan.item_node.size() : size_t(c->tree[sd].nnodes);
        if (v.rank.size() != n || v.nrows.size() != n || v.piv.size() != n * size_t(c->maxrank) ||
            v.xoff.size() != n + 1 || v.xoff.back() != int64_t(v.X.size()))
            throw Failure(NCA_ERR_ARG, "nca_core_load: inconsistent skeleton");
    }
    CK(cudaSetDevice(device));
    set_kernel_params(c.get(), &kd, c->tree[0].npoints, c->tree[1].npoints, nullptr);
    nca_build_opts o{};
    o.maxrank = c->maxrank;
    o.device = device;
    o.store_f32 = c->f32;
    o.compressor = dir ? NCA_COMPRESSOR_BOTTOMUP_IACA : NCA_COMPRESSOR_BATCHED_ACA;
    if (dir)
        build_dir_core(c.get(), pts[0].data(), pts[1].data(), &o, c->wb, &sv);
    else
        build_core(c.get(), pts[0].data(), c->tree[0].npoints, pts[1].data(), c->tree[1].npoints, &o, &sv);
    return c.release();
}

extern "C" {

int32_t nca_version(void) { return 2; }

int32_t nca_last_error(char *buf, size_t len) {
    if (!buf || len == 0) return NCA_ERR_ARG;
    size_t n = std::min(len - 1, g_error.size());
    std::memcpy(buf, g_error.data(), n);
    buf[n] = '\0';
    return NCA_OK;
}

int32_t nca_last_singular(int32_t *side, int32_t *node, int32_t *npivots, int32_t *rank) {
    *side = g_singular[0];
    *node = g_singular[1];
    *npivots = g_singular[2];
    *rank = g_singular[3];
    return NCA_OK;
}

int32_t nca_tree_kmeans(const double *points, int64_t npoints, int32_t minvalues, int32_t nclusters,
                        nca_tree **out) {
    return guarded([&] {
        if (!out || (npoints > 0 && !points)) return fail(NCA_ERR_ARG, "null argument");
        if (nclusters != 2) return fail(NCA_ERR_ARG, "only numberofclusters = 2 is supported");
        if (minvalues < 1) return fail(NCA_ERR_ARG, "minvalues must be positive");
        if (npoints >= (int64_t(1) << 31)) return fail(NCA_ERR_ARG, "too many points for 32-bit indices");
        // NCA_TREE_DEVICE=1: on the current CUDA device (bit for bit the host planner's tree). Not
        // the default: on 16 host cores the host planner builds the 262,144-point sphere's tree in
        // 0.047 s, the device in 0.14 s (one CTA per cluster: the top levels' ordered chunk sums
        // run on few SMs)
        int ndev = 0;
        const char *dv = std::getenv("NCA_TREE_DEVICE");
        const bool device = dv && std::strcmp(dv, "1") == 0 && cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0;
        cudaGetLastError();  // no device: not an error here
        auto t = std::make_unique<nca_tree>();
        if (device) {
            cudaStream_t s;
            CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
            struct StreamGuard {
                cudaStream_t s;
                ~StreamGuard() { cudaStreamDestroy(s); }
            } sg{s};
            t->t = build_kmeans_tree_device(points, npoints, minvalues, s);
        } else {
            t->t = build_kmeans_tree(points, npoints, minvalues);
        }
        *out = t.release();
        return int(NCA_OK);
    });
}

void nca_tree_destroy(nca_tree *tree) { delete tree; }

int32_t nca_tree_sizes(const nca_tree *tree, int32_t *nnodes, int32_t *nlevels, int64_t *npoints) {
    if (!tree) return fail(NCA_ERR_ARG, "null tree");
    *nnodes = tree->t.nnodes;
    *nlevels = tree->t.nlevels;
    *npoints = tree->t.npoints;
    return NCA_OK;
}

int32_t nca_tree_export(const nca_tree *tree, int32_t *perm, int32_t *begin, int32_t *end,
                        int32_t *parent, int32_t *firstchild, int32_t *nchildren, int32_t *level,
                        double *center, double *radius) {
    if (!tree) return fail(NCA_ERR_ARG, "null tree");
    const nca::Tree &T = tree->t;
    std::copy(T.perm.begin(), T.perm.end(), perm);
    std::copy(T.begin.begin(), T.begin.end(), begin);
    std::copy(T.end.begin(), T.end.end(), end);
    std::copy(T.parent.begin(), T.parent.end(), parent);
    std::copy(T.firstchild.begin(), T.firstchild.end(), firstchild);
    std::copy(T.nchildren.begin(), T.nchildren.end(), nchildren);
    std::copy(T.level.begin(), T.level.end(), level);
    std::copy(T.center.begin(), T.center.end(), center);
    std::copy(T.radius.begin(), T.radius.end(), radius);
    return NCA_OK;
}

int32_t nca_interactions(const nca_tree *test, const nca_tree *trial, double eta, nca_partition **out) {
    return guarded([&] {
        if (!test || !trial || !out) return fail(NCA_ERR_ARG, "null argument");
        auto *p = new nca_partition;
        p->p = build_partition(test->t, trial->t, eta);
        *out = p;
        return int(NCA_OK);
    });
}

int32_t nca_interactions_wideband(const nca_tree *test, const nca_tree *trial, double k, double etalf,
                                  double etahf, double gamma, nca_partition **out) {
    return guarded([&] {
        if (!test || !trial || !out) return fail(NCA_ERR_ARG, "null argument");
        if (!(k >= 0.0) || !(etalf > 0.0) || !(etahf > 0.0) || !(gamma > 0.0))
            return fail(NCA_ERR_ARG, "isnearwideband needs k >= 0 and positive eta_lf, eta_hf, gamma");
        auto *p = new nca_partition;
        p->wideband = true;
        p->w = nca::Wideband{k, etalf, etahf, gamma};
        p->p = build_partition_wideband(test->t, trial->t, p->w);
        *out = p;
        return int(NCA_OK);
    });
}

int32_t nca_directional_plan(const nca_tree *tree, const nca_tree *fartree, const nca_partition *part,
                             int32_t side, nca_dirplan **out) {
    return guarded([&] {
        if (!tree || !fartree || !part || !out || side < 0 || side > 1) return fail(NCA_ERR_ARG, "bad argument");
        if (!part->wideband) return fail(NCA_ERR_ARG, "directional plans need a wideband partition");
        const nca::Partition &P = part->p;
        const auto &ptr = side == 0 ? P.farptr : P.tfarptr;
        const auto &nodes = side == 0 ? P.farnodes : P.tfarnodes;
        if (int64_t(ptr.size()) != tree->t.nnodes + 1) return fail(NCA_ERR_DIM, "partition does not match the tree");
        auto *d = new nca_dirplan;
        d->tree = &tree->t;
        d->d = directional_plan(tree->t, fartree->t, ptr, nodes, part->w);
        *out = d;
        return int(NCA_OK);
    });
}

void nca_dirplan_destroy(nca_dirplan *plan) { delete plan; }

int32_t nca_dirplan_sizes(const nca_dirplan *plan, int32_t *nitems, int64_t *nfar, int64_t *nchildren) {
    if (!plan || !nitems || !nfar || !nchildren) return fail(NCA_ERR_ARG, "null argument");
    *nitems = int32_t(plan->d.item_node.size());
    *nfar = int64_t(plan->d.farnodes.size());
    *nchildren = int64_t(plan->d.item_chidx.size());
    return NCA_OK;
}

int32_t nca_dirplan_export(const nca_dirplan *plan, int32_t *farnodes, int32_t *dirptr, int32_t *dirs, double *dirvec,
                           int32_t *dirfarptr, int32_t *item_basis, int32_t *item_chptr, int32_t *item_chidx) {
    if (!plan) return fail(NCA_ERR_ARG, "null plan");
    const nca::DirSide &D = plan->d;
    std::copy(D.farnodes.begin(), D.farnodes.end(), farnodes);
    std::copy(D.dirptr.begin(), D.dirptr.end(), dirptr);
    std::copy(D.dirs.begin(), D.dirs.end(), dirs);
    std::copy(D.dirvec.begin(), D.dirvec.end(), dirvec);
    std::copy(D.dirfarptr.begin(), D.dirfarptr.end(), dirfarptr);
    std::copy(D.item_basis.begin(), D.item_basis.end(), item_basis);
    std::copy(D.item_chptr.begin(), D.item_chptr.end(), item_chptr);
    std::copy(D.item_chidx.begin(), D.item_chidx.end(), item_chidx);
    return NCA_OK;
}

int32_t nca_dirplan_farfield(const nca_dirplan *plan, int32_t item, int32_t *out, int32_t cap, int32_t *n) {
    return guarded([&] {
        if (!plan || !n || item < 0 || item >= int32_t(plan->d.item_node.size())) return fail(NCA_ERR_ARG, "bad argument");
        std::vector<int32_t> ff;
        item_farfield(*plan->tree, plan->d, item, ff);
        *n = int32_t(ff.size());
        if (out) std::copy(ff.begin(), ff.begin() + std::min<size_t>(ff.size(), size_t(std::max(cap, 0))), out);
        return int(NCA_OK);
    });
}

void nca_partition_destroy(nca_partition *part) { delete part; }

int32_t nca_partition_sizes(const nca_partition *part, int64_t *nnear, int64_t *nfar) {
    if (!part) return fail(NCA_ERR_ARG, "null partition");
    *nnear = int64_t(part->p.nearnodes.size());
    *nfar = int64_t(part->p.farnodes.size());
    return NCA_OK;
}

int32_t nca_partition_export(const nca_partition *part, int32_t *nearptr, int32_t *nearnodes,
                             int32_t *farptr, int32_t *farnodes, int32_t *trialfarptr,
                             int32_t *trialfarnodes) {
    if (!part) return fail(NCA_ERR_ARG, "null partition");
    const nca::Partition &P = part->p;
    std::copy(P.nearptr.begin(), P.nearptr.end(), nearptr);
    std::copy(P.nearnodes.begin(), P.nearnodes.end(), nearnodes);
    std::copy(P.farptr.begin(), P.farptr.end(), farptr);
    std::copy(P.farnodes.begin(), P.farnodes.end(), farnodes);
    std::copy(P.tfarptr.begin(), P.tfarptr.end(), trialfarptr);
    std::copy(P.tfarnodes.begin(), P.tfarnodes.end(), trialfarnodes);
    return NCA_OK;
}

int32_t nca_select_farpivots(const nca_tree *fartree, const double *ownpoints, const double *farpoints,
                             const int32_t *refidcs, int32_t nref, const int32_t *farnodes, int32_t nfar,
                             int32_t maxrank, int32_t *pivots, int32_t *npivots) {
    return guarded([&] {
        if (!fartree || !npivots) return fail(NCA_ERR_ARG, "null argument");
        if (maxrank < 0) return fail(NCA_ERR_ARG, "maxrank must be non-negative");
        for (int i = 0; i < nfar; ++i)
            if (farnodes[i] < 0 || farnodes[i] >= fartree->t.nnodes) return fail(NCA_ERR_ARG, "far node out of range");
        *npivots = select_farpivots(fartree->t, ownpoints, farpoints, refidcs, nref, farnodes, nfar, maxrank, pivots);
        return int(NCA_OK);
    });
}

int32_t nca_core_build(const double *testpoints, int64_t ntest, const double *trialpoints, int64_t ntrial,
                       const nca_tree *testtree, const nca_tree *trialtree, const nca_partition *part,
                       const nca_kernel_desc *kernel, const nca_build_opts *opts, nca_core **out) {
    return guarded([&] {
        if (!testtree || !trialtree || !part || !kernel || !opts || !out) return fail(NCA_ERR_ARG, "null argument");
        if (testtree->t.npoints != ntest || trialtree->t.npoints != ntrial)
            return fail(NCA_ERR_DIM, "DimensionMismatch: tree and point counts differ");
        if (opts->maxrank < 1 || opts->maxrank > 128) return fail(NCA_ERR_ARG, "maxrank must be in 1..128");
        if (!(opts->tol_test >= 0.0) || !(opts->tol_trial >= 0.0)) return fail(NCA_ERR_ARG, "tolerances must be non-negative");
        if (opts->compressor != NCA_COMPRESSOR_BATCHED_ACA && opts->compressor != NCA_COMPRESSOR_BOTTOMUP_IACA)
            return fail(NCA_ERR_ARG, "unknown compressor");
        if (part->wideband && opts->compressor != NCA_COMPRESSOR_BOTTOMUP_IACA)
            return fail(NCA_ERR_ARG, "Wideband (directional) NCA is only supported with BottomUp; got BatchedBottomUp "
                                     "as test compressor.");
        if (int64_t(part->p.nearptr.size()) != testtree->t.nnodes + 1 ||
            int64_t(part->p.tfarptr.size()) != trialtree->t.nnodes + 1)
            return fail(NCA_ERR_DIM, "partition does not match the trees");
        CK(cudaSetDevice(opts->device));
        auto c = std::make_unique<nca_core>();
        c->device = opts->device;
        c->maxrank = opts->maxrank;
        c->f32 = opts->store_f32 != 0;
        c->tree[0] = testtree->t;
        c->tree[1] = trialtree->t;
        c->part = part->p;
        set_kernel_params(c.get(), kernel, ntest, ntrial, nullptr);
        if (part->wideband) {
            c->wb = part->w;
            build_dir_core(c.get(), testpoints, trialpoints, opts, part->w);
        }
        else
            build_core(c.get(), testpoints, ntest, trialpoints, ntrial, opts);
        *out = c.release();
        return int(NCA_OK);
    });
}

void nca_core_destroy(nca_core *core) {
    if (!core) return;
    cudaSetDevice(core->device);
    delete core;
}

int32_t nca_core_save(const nca_core *core, const char *path) {
    if (!core || !path) return fail(NCA_ERR_ARG, "null argument");
    return guarded([&] {
        save_core(core, path);
        return int(NCA_OK);
    });
}

int32_t nca_core_load(const char *path, int32_t device, nca_core **out) {
    if (!path || !out) return fail(NCA_ERR_ARG, "null argument");
    return guarded([&] {
        *out = load_core(path, device);
        return int(NCA_OK);
    });
}

int32_t nca_core_set_wavenumber(nca_core *core, double k) {
    return guarded([&] {
        if (!core) return fail(NCA_ERR_ARG, "null core");
        if (core->moved) return fail(NCA_ERR_ARG, "the core's stores were moved into a batch");
        if (core->batch) return fail(NCA_ERR_ARG, "a batch has one wavenumber per member: refill the members");
        if (core->K.kind == NCA_KERNEL_MATRIX) return fail(NCA_ERR_ARG, "a matrix kernel has no wavenumber");
        if (!std::isfinite(k)) return fail(NCA_ERR_ARG, "the wavenumber must be finite");
        CK(cudaSetDevice(core->device));
        cudaStream_t s;
        CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        struct StreamGuard {
            cudaStream_t s;
            ~StreamGuard() { cudaStreamDestroy(s); }
        } sg{s};
        if (core->dir) {
            set_dir_wavenumber(core, k, s);
            return int(NCA_OK);
        }
        KernelParams K = core->K;
        K.k = k;
        K.deriv = 0;
        // new bases first (a singular frozen cross matrix leaves the core unchanged)
        DBuf<double2> X[2], XT[2];
        for (int sd = 0; sd < 2; ++sd) {
            X[sd].alloc(core->side[sd].X.n);
            XT[sd].alloc(core->side[sd].X.n);
            fill_bases(core, sd, 0, K, K, X[sd].p, XT[sd].p, s);
        }
        for (int sd = 0; sd < 2; ++sd) {
            std::swap(core->side[sd].X.p, X[sd].p);
            std::swap(core->side[sd].XT.p, XT[sd].p);
            core->side[sd].dX.release();
            core->side[sd].dXT.release();
        }
        core->K.k = k;
        fill_couplings(core, K, core->C.p, core->CT.p, s);
        fill_near(core, K, core->N.p, core->NT.p, s);
        if (core->f32) make_f32_copies(core, s);
        core->dC.release();
        core->dCT.release();
        core->dN.release();
        core->dNT.release();
        core->has_dk = false;
        CK(cudaStreamSynchronize(s));
        return int(NCA_OK);
    });
}

int32_t nca_core_prepare_dk(nca_core *core) {
    return guarded([&] {
        if (!core) return fail(NCA_ERR_ARG, "null core");
        if (core->moved) return fail(NCA_ERR_ARG, "the core's stores were moved into a batch");
        if (core->batch) return fail(NCA_ERR_ARG, "prepare the d/dk stores of the members, not of a batch");
        if (core->K.kind == NCA_KERNEL_MATRIX) return fail(NCA_ERR_ARG, "a matrix kernel has no wavenumber derivative");
        if (core->has_dk) return int(NCA_OK);
        CK(cudaSetDevice(core->device));
        cudaStream_t s;
        CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        struct StreamGuard {
            cudaStream_t s;
            ~StreamGuard() { cudaStreamDestroy(s); }
        } sg{s};
        if (core->dir) {
            prepare_dir_dk(core, s);
            return int(NCA_OK);
        }
        KernelParams dK = core->K;
        dK.deriv = 1;
        for (int sd = 0; sd < 2; ++sd) {
            DevSide &d = core->side[sd];
            d.dX.alloc(d.X.n);
            d.dXT.alloc(d.X.n);
            fill_bases(core, sd, 1, core->K, dK, d.dX.p, d.dXT.p, s);
        }
        core->dC.alloc(core->C.n);
        core->dCT.alloc(core->CT.n);
        fill_couplings(core, dK, core->dC.p, core->dCT.p, s);
        core->dN.alloc(core->N.n);
        core->dNT.alloc(core->NT.n);
        fill_near(core, dK, core->dN.p, core->dNT.p, s);
        CK(cudaStreamSynchronize(s));
        core->has_dk = true;
        return int(NCA_OK);
    });
}

int32_t nca_core_batch(nca_core *const *cores, int32_t ncores, int32_t flags, nca_core **out) {
    return guarded([&] {
        if (!cores || !out || ncores < 1) return fail(NCA_ERR_ARG, "a batch needs at least one core");
        if (flags & ~int32_t(NCA_BATCH_MOVE_STORES)) return fail(NCA_ERR_ARG, "unknown batch flags");
        std::vector<nca_core *> cs(cores, cores + ncores);
        int64_t nt = 0, ns = 0;
        for (size_t i = 0; i < cs.size(); ++i) {
            const nca_core *c = cs[i];
            if (!c) return fail(NCA_ERR_ARG, "null core in the batch");
            if (c->moved) return fail(NCA_ERR_ARG, "a core of the batch was moved into another batch");
            if (c->dir) return fail(NCA_ERR_ARG, "directional cores cannot be batched");
            for (size_t j = 0; j < i; ++j)
                if (cs[j] == c) return fail(NCA_ERR_ARG, "a core appears twice in the batch");
            if (c->device != cs[0]->device) return fail(NCA_ERR_ARG, "the cores of a batch must share one device");
            nt += c->side[0].npts;
            ns += c->side[1].npts;
        }
        if (nt >= (int64_t(1) << 31) || ns >= (int64_t(1) << 31))
            return fail(NCA_ERR_ARG, "too many points in the batch for 32-bit indices");
        CK(cudaSetDevice(cs[0]->device));
        auto m = std::make_unique<nca_core>();
        merge_core(cs, m.get(), (flags & NCA_BATCH_MOVE_STORES) != 0, nullptr);
        CK(cudaStreamSynchronize(nullptr));
        *out = m.release();
        return int(NCA_OK);
    });
}

int32_t nca_core_get_info(const nca_core *core, nca_core_info *info) {
    if (!core || !info) return fail(NCA_ERR_ARG, "null argument");
    *info = core->info;
    return NCA_OK;
}

int32_t nca_core_export_pivots(const nca_core *core, int32_t side, int32_t *ranks, int32_t *nrows,
                               int32_t *ptr, int32_t *idx) {
    if (!core || side < 0 || side > 1) return fail(NCA_ERR_ARG, "bad argument");
    if (core->dir) return fail(NCA_ERR_ARG, "node exports are not available for directional cores");
    const DevSide &d = core->side[side];
    int nn = d.nnodes;
    std::copy(d.h_rank.begin(), d.h_rank.end(), ranks);
    std::copy(d.h_nrows.begin(), d.h_nrows.end(), nrows);
    ptr[0] = 0;
    for (int t = 0; t < nn; ++t) {
        ptr[t + 1] = ptr[t] + d.h_rank[t];
        std::copy(d.h_piv.begin() + int64_t(t) * core->maxrank,
                  d.h_piv.begin() + int64_t(t) * core->maxrank + d.h_rank[t], idx + ptr[t]);
    }
    return NCA_OK;
}

int32_t nca_core_dir_items(const nca_core *core, int32_t side, int32_t *nitems, int32_t *ranks, int32_t *nrows,
                           int32_t *ptr, int32_t *idx) {
    if (!core || side < 0 || side > 1 || !nitems) return fail(NCA_ERR_ARG, "bad argument");
    if (!core->dir) return fail(NCA_ERR_ARG, "not a directional core");
    const DirItems &d = core->dir->side[side];
    *nitems = d.nitems;
    if (!ranks) return NCA_OK;
    return guarded([&] {
        CK(cudaSetDevice(core->device));
        const std::vector<int32_t> piv = download_now(d.piv, size_t(d.nitems) * core->maxrank);
        std::copy(d.h_rank.begin(), d.h_rank.end(), ranks);
        std::copy(d.h_nrows.begin(), d.h_nrows.end(), nrows);
        ptr[0] = 0;
        for (int it = 0; it < d.nitems; ++it) {
            ptr[it + 1] = ptr[it] + d.h_rank[it];
            std::copy(piv.begin() + int64_t(it) * core->maxrank, piv.begin() + int64_t(it) * core->maxrank + d.h_rank[it],
                      idx + ptr[it]);
        }
        return int(NCA_OK);
    });
}

int32_t nca_core_farpivots_total(const nca_core *core, int32_t side, int64_t *total) {
    if (!core || side < 0 || side > 1) return fail(NCA_ERR_ARG, "bad argument");
    if (core->dir) return fail(NCA_ERR_ARG, "node exports are not available for directional cores");
    *total = core->side[side].h_fpptr.back();
    return NCA_OK;
}

int32_t nca_core_export_farpivots(const nca_core *core, int32_t side, int32_t *ptr, int32_t *idx) {
    if (!core || side < 0 || side > 1) return fail(NCA_ERR_ARG, "bad argument");
    if (core->dir) return fail(NCA_ERR_ARG, "node exports are not available for directional cores");
    const DevSide &d = core->side[side];
    std::copy(d.h_fpptr.begin(), d.h_fpptr.end(), ptr);
    std::copy(d.h_fpidx.begin(), d.h_fpidx.end(), idx);
    return NCA_OK;
}

int32_t nca_core_export_x(const nca_core *core, int32_t side, int64_t *off, double *X) {
    return guarded([&] {
        if (!core || side < 0 || side > 1) return fail(NCA_ERR_ARG, "bad argument");
        if (core->moved) return fail(NCA_ERR_ARG, "the core's stores were moved into a batch");
        if (core->dir) return fail(NCA_ERR_ARG, "node exports are not available for directional cores");
        const DevSide &d = core->side[side];
        CK(cudaSetDevice(core->device));
        std::vector<double2> all(d.X.n);
        if (d.X.n) CK(cudaMemcpy(all.data(), d.X.p, sizeof(double2) * d.X.n, cudaMemcpyDeviceToHost));
        off[0] = 0;
        for (int t = 0; t < d.nnodes; ++t) {
            int64_t e = int64_t(d.h_nrows[t]) * d.h_rank[t];
            off[t + 1] = off[t] + e;
            std::memcpy(X + 2 * off[t], all.data() + d.h_xoff[t], sizeof(double2) * e);
        }
        return int(NCA_OK);
    });
}

int32_t nca_core_export_couplings(const nca_core *core, int64_t *off, double *C) {
    return guarded([&] {
        if (!core) return fail(NCA_ERR_ARG, "null core");
        if (core->moved) return fail(NCA_ERR_ARG, "the core's stores were moved into a batch");
        if (core->dir) return fail(NCA_ERR_ARG, "node exports are not available for directional cores");
        CK(cudaSetDevice(core->device));
        std::vector<double2> all(core->C.n);
        if (core->C.n) CK(cudaMemcpy(all.data(), core->C.p, sizeof(double2) * core->C.n, cudaMemcpyDeviceToHost));
        const nca::Partition &P = core->part;
        off[0] = 0;
        for (int t = 0; t < core->tree[0].nnodes; ++t)
            for (int i = P.farptr[t]; i < P.farptr[t + 1]; ++i) {
                const int64_t e = int64_t(core->side[0].h_rank[t]) * core->side[1].h_rank[P.farnodes[i]];
                off[i + 1] = off[i] + e;
                std::memcpy(C + 2 * off[i], all.data() + core->h_cfoff[i], sizeof(double2) * e);
            }
        return int(NCA_OK);
    });
}

int32_t nca_core_export_near(const nca_core *core, int64_t *off, int32_t *ncols, double *N) {
    return guarded([&] {
        if (!core) return fail(NCA_ERR_ARG, "null core");
        if (core->moved) return fail(NCA_ERR_ARG, "the core's stores were moved into a batch");
        CK(cudaSetDevice(core->device));
        std::vector<double2> all(core->N.n);
        if (core->N.n) CK(cudaMemcpy(all.data(), core->N.p, sizeof(double2) * core->N.n, cudaMemcpyDeviceToHost));
        const nca::Partition &P = core->part;
        std::copy(core->h_noff.begin(), core->h_noff.end(), off);
        std::copy(core->h_ncols.begin(), core->h_ncols.end(), ncols);
        for (int t = 0; t < core->tree[0].nnodes; ++t) {
            int64_t pos = core->h_noff[t];
            for (int i = P.nearptr[t]; i < P.nearptr[t + 1]; ++i) {
                const int64_t e = int64_t(core->tree[0].size(t)) * core->tree[1].size(P.nearnodes[i]);
                std::memcpy(N + 2 * pos, all.data() + core->h_nfoff[i], sizeof(double2) * e);
                pos += e;
            }
        }
        return int(NCA_OK);
    });
}

int32_t nca_workspace_create(nca_core *core, int32_t max_nrhs, nca_workspace **out) {
    return guarded([&] {
        if (!core || !out) return fail(NCA_ERR_ARG, "null argument");
        if (core->moved) return fail(NCA_ERR_ARG, "the core's stores were moved into a batch");
        CK(cudaSetDevice(core->device));
        auto ws = std::make_unique<nca_workspace>();
        ws->core = core;
        CK(cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking));
        CK(cudaEventCreate(&ws->e0));
        CK(cudaEventCreate(&ws->e1));
        if (!core->dir) {
            int least = 0, greatest = 0;
            CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
            CK(cudaStreamCreateWithPriority(&ws->aux, cudaStreamNonBlocking, greatest));
            ws->aux_priority = greatest;
            CK(cudaEventCreateWithFlags(&ws->fork, cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&ws->join, cudaEventDisableTiming));
        }
        int b = std::max(1, max_nrhs);
        if (!core->dir) {
            ws->xt.alloc(size_t(std::max(core->side[0].npts, core->side[1].npts)) * vector_slots(b));
            ws->xhat.alloc(size_t(std::max(core->side[0].h_cptr.back(), core->side[1].h_cptr.back())) * vector_slots(b));
            ws->yhat.alloc(ws->xhat.n);
        }
        ws->max_nrhs = b;
        ws->error.alloc(1);
        CK(cudaMallocHost(&ws->error_host, sizeof(int32_t)));
        *out = ws.release();
        return int(NCA_OK);
    });
}

void nca_workspace_destroy(nca_workspace *ws) {
    if (!ws) return;
    cudaSetDevice(ws->core->device);
    drop_graphs(ws);
    if (ws->stream) cudaStreamDestroy(ws->stream);
    if (ws->aux) cudaStreamDestroy(ws->aux);
    if (ws->fork) cudaEventDestroy(ws->fork);
    if (ws->join) cudaEventDestroy(ws->join);
    if (ws->e0) cudaEventDestroy(ws->e0);
    if (ws->e1) cudaEventDestroy(ws->e1);
    for (cudaEvent_t &e : ws->stage_ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : ws->dir_ev) cudaEventDestroy(e);
    if (ws->error_host) cudaFreeHost(ws->error_host);
    delete ws;
}

int32_t nca_workspace_autotune(nca_workspace *ws, int32_t mode, int32_t precision, int64_t nrhs, int32_t *choice) {
    if (!ws) return fail(NCA_ERR_ARG, "null workspace");
    bool expected = false;
    if (!ws->busy.compare_exchange_strong(expected, true))
        return fail(NCA_ERR_BUSY, "ConcurrentWorkspaceError: the workspace is in use by another matrix-vector product");
    int st = guarded([&] {
        nca_core *c = ws->core;
        if (nrhs < 1) return fail(NCA_ERR_ARG, "nrhs must be positive");
        if (mode < 0 || mode > 2) return fail(NCA_ERR_ARG, "mode must be 0 (N), 1 (T) or 2 (C)");
        CK(cudaSetDevice(c->device));
        const int in = mode == 0 ? 1 : 0, out = 1 - in;
        const int64_t nin = c->side[in].npts, nout = c->side[out].npts;
        DBuf<double2> xd, yd;
        xd.alloc(size_t(nin) * nrhs);
        yd.alloc(size_t(nout) * nrhs);
        xd.zero(ws->stream);
        yd.zero(ws->stream);
        const bool profiling = ws->profiling;
        ws->profiling = false;
        // schedules: (overlap of the near field with the sweeps, CUDA-graph replay); directional
        // cores have no second stream
        const int nconf = c->dir ? 2 : 4;
        double best = 1e30;
        int arg = 0;
        for (int k = 0; k < nconf; ++k) {
            ws->use_overlap = c->dir ? false : (k & 1) == 0;
            ws->use_graphs = (k & 2) != 0 || (c->dir && k == 1);
            drop_graphs(ws);
            double tsum = 0.0;
            for (int rep = 0; rep < 8; ++rep) {
                if (int e = apply_impl(ws, mode, precision, xd.p, nin, yd.p, nout, nrhs, make_double2(1.0, 0.0),
                                       make_double2(0.0, 0.0), 1))
                    return e;
                if (rep >= 3) tsum += ws->last_seconds;  // three calls warm up (and capture a graph)
            }
            if (tsum < best) {
                best = tsum;
                arg = k;
            }
        }
        ws->use_overlap = c->dir ? false : (arg & 1) == 0;
        ws->use_graphs = (arg & 2) != 0 || (c->dir && arg == 1);
        drop_graphs(ws);
        ws->profiling = profiling;
        if (choice) *choice = (ws->use_overlap ? 1 : 0) | (ws->use_graphs ? 2 : 0);
        return int(NCA_OK);
    });
    ws->busy.store(false);
    return st;
}

int32_t nca_apply(nca_workspace *ws, int32_t mode, int32_t precision, const void *x, int64_t ldx, void *y,
                  int64_t ldy, int64_t nrhs, double alpha_re, double alpha_im, double beta_re, double beta_im,
                  int32_t memspace) {
    if (!ws) return fail(NCA_ERR_ARG, "null workspace");
    bool expected = false;
    if (!ws->busy.compare_exchange_strong(expected, true))
        return fail(NCA_ERR_BUSY, "ConcurrentWorkspaceError: the workspace is in use by another matrix-vector product");
    int st = guarded([&] {
        return apply_impl(ws, mode, precision, x, ldx, y, ldy, nrhs, make_double2(alpha_re, alpha_im),
                          make_double2(beta_re, beta_im), memspace);
    });
    ws->busy.store(false);
    return st;
}

int32_t nca_apply_static(nca_core *core, int32_t mode, int32_t precision, const void *x, int64_t ldx, void *y,
                         int64_t ldy, int64_t nrhs, double alpha_re, double alpha_im, double beta_re,
                         double beta_im, void *stream) {
    if (!core) return fail(NCA_ERR_ARG, "null core");
    return guarded([&] {
        return apply_static_impl(core, mode, precision, x, ldx, y, ldy, nrhs, make_double2(alpha_re, alpha_im),
                                 make_double2(beta_re, beta_im), static_cast<cudaStream_t>(stream));
    });
}

int32_t nca_apply_dk(nca_workspace *ws, const void *x, int64_t ldx, void *y, int64_t ldy, int64_t nrhs,
                     double alpha_re, double alpha_im, double beta_re, double beta_im, int32_t memspace) {
    if (!ws) return fail(NCA_ERR_ARG, "null workspace");
    bool expected = false;
    if (!ws->busy.compare_exchange_strong(expected, true))
        return fail(NCA_ERR_BUSY, "ConcurrentWorkspaceError: the workspace is in use by another matrix-vector product");
    int st = guarded([&] {
        return apply_impl(ws, 0, NCA_PREC_F64, x, ldx, y, ldy, nrhs, make_double2(alpha_re, alpha_im),
                          make_double2(beta_re, beta_im), memspace, true);
    });
    ws->busy.store(false);
    return st;
}

int32_t nca_workspace_last_time(const nca_workspace *ws, double *seconds) {
    if (!ws || !seconds) return fail(NCA_ERR_ARG, "null argument");
    *seconds = ws->last_seconds;
    return NCA_OK;
}

int32_t nca_workspace_last_launches(const nca_workspace *ws, int32_t *launches) {
    if (!ws || !launches) return fail(NCA_ERR_ARG, "null argument");
    *launches = ws->last_launches;
    return NCA_OK;
}

int32_t nca_workspace_set_parts(nca_workspace *ws, int32_t far, int32_t near) {
    if (!ws) return fail(NCA_ERR_ARG, "null workspace");
    ws->far = far != 0;
    ws->near = near != 0;
    return NCA_OK;
}

int32_t nca_workspace_set_graphs(nca_workspace *ws, int32_t on) {
    return guarded([&] {
        if (!ws) return fail(NCA_ERR_ARG, "null workspace");
        CK(cudaSetDevice(ws->core->device));
        if (!on) drop_graphs(ws);
        ws->use_graphs = on != 0;
        return int(NCA_OK);
    });
}

int32_t nca_workspace_set_profiling(nca_workspace *ws, int32_t on) {
    return guarded([&] {
        if (!ws) return fail(NCA_ERR_ARG, "null workspace");
        CK(cudaSetDevice(ws->core->device));
        for (cudaEvent_t &e : ws->stage_ev)
            if (!e) CK(cudaEventCreate(&e));
        ws->profiling = on != 0;
        return int(NCA_OK);
    });
}

int32_t nca_workspace_stage_times(const nca_workspace *ws, double *seconds, int32_t *launches, int32_t nstages) {
    if (!ws || nstages < 0) return fail(NCA_ERR_ARG, "bad argument");
    for (int k = 0; k < std::min(nstages, kStages); ++k) {
        if (seconds) seconds[k] = ws->stage_seconds[k];
        if (launches) launches[k] = ws->stage_launches[k];
    }
    return NCA_OK;
}

int32_t nca_blocks_aca(const double *buffer, int64_t ldbuffer, int32_t ldcols, const int64_t *rowoffsets,
                       const int32_t *ncols, int32_t nblocks, int32_t maxrank, double tol, int32_t sampled,
                       int32_t device, int32_t *ranks, int32_t *rowpivots, int32_t *colpivots) {
    return guarded([&] {
        if (nblocks < 0 || maxrank < 1 || maxrank > 128) return fail(NCA_ERR_ARG, "bad block arguments");
        if (nblocks == 0) return int(NCA_OK);
        CK(cudaSetDevice(device));
        int mcap = 0, ncap = 1;
        for (int i = 0; i < nblocks; ++i) {
            mcap = std::max<int>(mcap, int(rowoffsets[i + 1] - rowoffsets[i]));
            if (ncols[i] > ldcols) return fail(NCA_ERR_ARG, "ncols exceeds the buffer width");
            ncap = std::max(ncap, ncols[i]);
        }
        mcap = std::max(mcap, 1);
        size_t sm = sizeof(double2) * (size_t(mcap) * ncap + mcap + ncap) + sizeof(int32_t) * 2 * ncap + 16;
        if (sm > size_t(kMaxSmem)) return fail(NCA_ERR_ARG, "block does not fit in shared memory");
        cudaStream_t s = nullptr;
        DBuf<double2> dbuf;
        dbuf.upload(reinterpret_cast<const double2 *>(buffer), size_t(ldbuffer) * ldcols, s);
        DBuf<int64_t> doff;
        doff.upload(rowoffsets, size_t(nblocks) + 1, s);
        DBuf<int32_t> dn, dr, drp, dcp;
        dn.upload(ncols, nblocks, s);
        dr.alloc(nblocks);
        drp.alloc(size_t(nblocks) * maxrank);
        dcp.alloc(size_t(nblocks) * maxrank);
        CK(cudaFuncSetAttribute(k_blocks_aca, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
        k_blocks_aca<<<nblocks, 256, sm, s>>>(dbuf.p, ldbuffer, doff.p, dn.p, maxrank, tol, sampled, mcap, ncap,
                                              dr.p, drp.p, dcp.p);
        CK(cudaGetLastError());
        CK(cudaMemcpy(ranks, dr.p, sizeof(int32_t) * nblocks, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(rowpivots, drp.p, sizeof(int32_t) * nblocks * maxrank, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(colpivots, dcp.p, sizeof(int32_t) * nblocks * maxrank, cudaMemcpyDeviceToHost));
        return int(NCA_OK);
    });
}

int32_t nca_blocks_factors(const double *buffer, int64_t ldbuffer, int32_t ldcols, const int64_t *rowoffsets,
                           int32_t nblocks, const int32_t *ranks, const int32_t *rowpivots,
                           const int32_t *colpivots, int32_t maxrank, int32_t device, const int64_t *zoff,
                           double *Z) {
    return guarded([&] {
        if (nblocks < 0 || maxrank < 1 || maxrank > 128) return fail(NCA_ERR_ARG, "bad block arguments");
        if (nblocks == 0) return int(NCA_OK);
        CK(cudaSetDevice(device));
        int mcap = 1;
        for (int i = 0; i < nblocks; ++i) {
            int m = int(rowoffsets[i + 1] - rowoffsets[i]);
            mcap = std::max(mcap, m);
            if (ranks[i] < 0 || ranks[i] > maxrank || ranks[i] > m) return fail(NCA_ERR_ARG, "rank out of range");
            for (int k = 0; k < ranks[i]; ++k) {
                int rp = rowpivots[int64_t(i) * maxrank + k], cp = colpivots[int64_t(i) * maxrank + k];
                if (rp < 0 || rp >= m || cp < 0 || cp >= ldcols) return fail(NCA_ERR_ARG, "pivot out of range");
            }
        }
        size_t sm = sizeof(double2) * size_t(maxrank) * maxrank + sizeof(int32_t) * maxrank + 16;
        if (sm > size_t(kMaxSmem)) return fail(NCA_ERR_ARG, "block does not fit in shared memory");
        cudaStream_t s = nullptr;
        DBuf<double2> dbuf, dz;
        dbuf.upload(reinterpret_cast<const double2 *>(buffer), size_t(ldbuffer) * ldcols, s);
        DBuf<int64_t> doff, dzoff;
        doff.upload(rowoffsets, size_t(nblocks) + 1, s);
        dzoff.upload(zoff, size_t(nblocks) + 1, s);
        DBuf<int32_t> dr, drp, dcp, st;
        dr.upload(ranks, nblocks, s);
        drp.upload(rowpivots, size_t(nblocks) * maxrank, s);
        dcp.upload(colpivots, size_t(nblocks) * maxrank, s);
        st.alloc(4);
        st.zero(s);
        dz.alloc(size_t(zoff[nblocks]));
        CK(cudaFuncSetAttribute(k_blocks_factors, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
        k_blocks_factors<<<nblocks, 256, sm, s>>>(dbuf.p, ldbuffer, doff.p, dr.p, drp.p, dcp.p, maxrank,
                                                  dzoff.p, dz.p, st.p);
        CK(cudaGetLastError());
        std::vector<int32_t> h = st.download(s);
        if (h[0] == 1) {
            set_singular(0, h[1], h[2], h[3]);
            return fail(NCA_ERR_SINGULAR, "SingularCrossMatrixError: block " + std::to_string(h[1]) + " has " +
                                              std::to_string(h[2]) + " pivots but rank " + std::to_string(h[3]));
        }
        if (dz.n) CK(cudaMemcpy(Z, dz.p, sizeof(double2) * dz.n, cudaMemcpyDeviceToHost));
        return int(NCA_OK);
    });
}

int32_t nca_entries(const nca_kernel_desc *kernel, const double *testpoints, int64_t ntest,
                    const double *trialpoints, int64_t ntrial, const int64_t *ii, const int64_t *jj, int64_t n,
                    int32_t device, double *out) {
    return entries_impl(kernel, testpoints, ntest, trialpoints, ntrial, ii, jj, n, device, out, 0);
}

int32_t nca_entries_dk(const nca_kernel_desc *kernel, const double *testpoints, int64_t ntest,
                       const double *trialpoints, int64_t ntrial, const int64_t *ii, const int64_t *jj, int64_t n,
                       int32_t device, double *out) {
    if (kernel && kernel->kind == NCA_KERNEL_MATRIX) return fail(NCA_ERR_ARG, "a matrix kernel has no wavenumber derivative");
    return entries_impl(kernel, testpoints, ntest, trialpoints, ntrial, ii, jj, n, device, out, 1);
}

}  // extern "C"

namespace {
int entries_impl(const nca_kernel_desc *kernel, const double *testpoints, int64_t ntest, const double *trialpoints,
                 int64_t ntrial, const int64_t *ii, const int64_t *jj, int64_t n, int32_t device, double *out,
                 int deriv) {
    return guarded([&] {
        if (!kernel || n < 0) return fail(NCA_ERR_ARG, "bad argument");
        if (n == 0) return int(NCA_OK);
        for (int64_t e = 0; e < n; ++e)
            if (ii[e] < 0 || ii[e] >= ntest || jj[e] < 0 || jj[e] >= ntrial) return fail(NCA_ERR_ARG, "index out of range");
        CK(cudaSetDevice(device));
        nca_core tmp;
        set_kernel_params(&tmp, kernel, ntest, ntrial, nullptr);
        DBuf<double> tp, sp;
        tp.upload(testpoints, size_t(3 * ntest), nullptr);
        sp.upload(trialpoints, size_t(3 * ntrial), nullptr);
        DBuf<int64_t> di, dj;
        di.upload(ii, size_t(n), nullptr);
        dj.upload(jj, size_t(n), nullptr);
        DBuf<double2> dout;
        dout.alloc(size_t(n));
        tmp.K.deriv = deriv;
        k_entries<<<launch_grid(n / 256 + 1, 8), 256>>>(tmp.K, tp.p, sp.p, di.p, dj.p, n, dout.p);
        CK(cudaGetLastError());
        CK(cudaMemcpy(out, dout.p, sizeof(double2) * n, cudaMemcpyDeviceToHost));
        return int(NCA_OK);
    });
}

}  // namespace

