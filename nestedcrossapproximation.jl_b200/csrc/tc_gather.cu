// STAGE_GATHER of the directional products over complex-FP32 stores and arena on the 5th-generation
// tensor cores (tcgen05, kind::tf32, operands in shared memory, accumulators in tensor memory).
//
// One output o of R <= 64 rows and all b right-hand sides (up to 128 per pass) is
//   out(R x b) = sum over segments e of M_e (R x w_e) V_e (w_e x b)     (complex).
// Viewed as real matrices with interleaved real and imaginary parts, the vector rows and the block
// columns are already the two operands of one real product:
//   A (M = 2 b, K) with A[2c + tv][j] = part tv of V[j][c]      (the vector row j, as stored)
//   B (N = 2 R, K) with B[2r + tm][j] = part tm of M[r][j]      (the block column j, as stored)
//   D = A B^T,     D[2c + tv][2r + tm] = sum_j V_tv[j][c] M_tm[r][j]
// and out[r][c] = (D[2c][2r] - D[2c+1][2r+1]) + i (D[2c][2r+1] + D[2c+1][2r]) (conjugated blocks:
// the signs of the M_i terms flip). M = 2 b runs over two 128-row tiles (64 right-hand sides each), N = 2 R is
// padded to a multiple of 16 (at most 128), K runs over the output's (block column, vector row)
// pairs, 16 per chunk and segment.
//
// Precision: every operand is split into a TF32 head (rounded to nearest) and the TF32-rounded
// remainder, and each k-step issues hi*hi + hi*lo + lo*hi into the FP32 accumulator (3xTF32), which
// leaves an error of about 2^-21 of each product, the class of FP32 arithmetic.
//
// Schedule: one CTA of 128 threads per output at a time (grid-stride over the outputs, two CTAs per
// SM). For each chunk all threads load its vector rows and block columns from global memory, split
// them and store the four operand tiles into one of two shared-memory stages (canonical
// no-swizzle K-major layout: core matrices of 8 rows x 4 k-elements, 128 bytes; the two 4-element
// k halves of a k-step 128 bytes apart, 8-row groups 256 bytes apart; the stored vectors and blocks
// are MN-contiguous, so each element is placed on its own); one thread issues the MMAs and commits
// them to the stage's mbarrier. The loads of
// the next chunk are issued before the previous output's epilogue (tensor memory to registers,
// real/imaginary combination through a lane shuffle, stores) so that their latency overlaps it.
// Waits on mbarriers are bounded: a wait that runs out sets error = 2 and the kernel finishes
// without further MMAs.
#include <cuda_runtime.h>

#include <cstdint>

#include "apply_kernels.cuh"

namespace nca {

namespace {

constexpr int TC_THREADS = 128;
constexpr int TC_KC = 16;            // pairs per chunk (two k-steps of 8)
constexpr int TC_TILE_A = 128 * 8 * 4;  // bytes of one 128 x 8 operand tile of A (one k-step)
constexpr int TC_TILE_B = 128 * 8 * 4;  // bytes of one (N <= 128) x 8 tile of B
// one stage: A hi/lo for 2 M tiles x 2 k-steps, B hi/lo for 2 k-steps
constexpr int TC_STAGE = 2 * (2 * 2 * TC_TILE_A) + 2 * (2 * TC_TILE_B);
constexpr int TC_SMEM = 2 * TC_STAGE + 64;  // two stages, then mbarriers and the tensor-memory base
constexpr unsigned kTcWaitLimit = 1u << 20;

__device__ __forceinline__ uint32_t su32(const void *p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// offsets inside a stage
__device__ __forceinline__ int a_off(int hl, int tile, int kg) { return ((hl * 2 + tile) * 2 + kg) * TC_TILE_A; }
__device__ __forceinline__ int b_off(int hl, int kg) { return 2 * (2 * 2 * TC_TILE_A) + (hl * 2 + kg) * TC_TILE_B; }

// shared-memory matrix descriptor, no swizzle, K-major: start address, leading-dimension byte
// offset (between the core matrices of a row group along k), stride byte offset (between 8-row
// groups), version 1
__device__ __forceinline__ uint64_t mdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= uint64_t((addr >> 4) & 0x3FFFu);
    d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
    d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
    d |= uint64_t(1) << 46;  // descriptor version
    return d;                 // base offset 0, swizzle none
}

// instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B, both K-major, M = 128
__device__ __forceinline__ uint32_t idesc_tf32(int n) {
    uint32_t d = 0;
    d |= 1u << 4;                     // D format F32
    d |= 2u << 7;                     // A format TF32
    d |= 2u << 10;                    // B format TF32
    d |= uint32_t(n >> 3) << 17;      // N / 8
    d |= uint32_t(128 >> 4) << 24;    // M / 16
    return d;
}

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(dtmem),
        "l"(a), "l"(b), "r"(idesc), "r"(uint32_t(accumulate))
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
                 : "memory");
}

__device__ __forceinline__ void bar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(bar)), "r"(count) : "memory");
}

// waits for the completion of phase `parity` of bar; false when the wait ran out
__device__ __forceinline__ bool bar_wait(uint64_t *bar, uint32_t parity) {
    for (unsigned it = 0; it < kTcWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(su32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ uint32_t tf32_round(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// head (rounded to TF32) and tail of x; the tail is passed as FP32 bits, whose low 13 bits the
// MMA ignores: it loses below 2^-10 of the tail, below 2^-21 of x
__device__ __forceinline__ void split(float x, uint32_t &hi, uint32_t &lo) {
    hi = tf32_round(x);
    lo = __float_as_uint(x - __uint_as_float(hi));
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// A chunk: segment e, its block columns / vector rows [j0, j0 + jn) (jn <= TC_KC), of one output pass
struct TcChunk {
    int wi, c0, e, j0, jn;
    bool first, last;  // first / last chunk of its (output, pass)
};

// Register-held loads of one chunk: thread (warp w, lane l) holds the A elements i = 0..31 and the
// B elements i = 0..15 with kq = l & 3, rq = l >> 2, rest = 4 i + w: k = 4 (rest & 3) + kq and
// row 8 (rest >> 2) + rq (A: one of the 2 x 128 tile rows; B: one of the 128). The 32 lanes of a
// warp store 32 distinct (row mod 8, k mod 4) positions: 32 different banks.
struct TcLoad {
    float a[32];
    float b[16];
};

// The CTA's walk over its outputs (grid-stride), their passes of 128 right-hand sides and the
// (block column, vector row) pairs of each pass, TC_KC pairs per chunk across segment boundaries:
// the chunk starts at pair j0 of segment e, t pairs of the pass are done. Every thread walks it
// identically.
struct TcWalk {
    int wi, c0, e, j0, w, t;
    WideOut rec;
};

__device__ __forceinline__ WideOut tc_record(const WideOut *outs, int i) {
    const int4 *q = reinterpret_cast<const int4 *>(outs + i);
    const int4 u = q[0], v = q[1];
    WideOut o;
    o.R = u.x;
    o.W = u.y;
    o.e0 = u.z;
    o.e1 = u.w;
    o.out = int64_t((uint64_t(uint32_t(v.y)) << 32) | uint32_t(v.x));
    o.ld = v.z;
    o.r0 = v.w;
    return o;
}

// the chunk the walk stands on: jn = 0 for a pass of an output without pairs (its outputs are
// written from zero); false once the walk is past the last output
__device__ __forceinline__ bool tc_chunk(const TcWalk &k, int count, TcChunk &ch) {
    if (k.wi >= count) return false;
    ch.wi = k.wi;
    ch.c0 = k.c0;
    ch.e = k.e;
    ch.j0 = k.j0;
    ch.jn = min(TC_KC, k.rec.W - k.t);
    ch.first = k.t == 0;
    ch.last = k.t + ch.jn >= k.rec.W;
    return true;
}

__device__ __forceinline__ void tc_pass_start(const RowArgs<float2> &a, TcWalk &k) {
    k.e = k.rec.e0;
    k.j0 = 0;
    k.t = 0;
    k.w = k.e < k.rec.e1 ? a.g_w[k.e] : 0;
}

__device__ __forceinline__ void tc_start_output(const RowArgs<float2> &a, const WideOut *outs, int count, TcWalk &k) {
    k.c0 = 0;
    if (k.wi >= count) return;
    k.rec = tc_record(outs, k.wi);
    tc_pass_start(a, k);
}

// moves the walk to the next chunk
__device__ __forceinline__ void tc_advance(const RowArgs<float2> &a, const WideOut *outs, int count, TcWalk &k) {
    int rem = min(TC_KC, k.rec.W - k.t);
    k.t += rem;
    if (k.t < k.rec.W) {
        while (rem > 0) {
            const int take = min(rem, k.w - k.j0);
            k.j0 += take;
            rem -= take;
            if (k.j0 >= k.w) {
                ++k.e;
                k.j0 = 0;
                k.w = a.g_w[k.e];  // e < e1: pairs remain
            }
        }
        return;
    }
    // the pass is done: the next pass of the output, or the next output
    k.c0 += 128;
    if (k.c0 < a.b) {
        tc_pass_start(a, k);
        return;
    }
    k.wi += gridDim.x;
    tc_start_output(a, outs, count, k);
}

// the chunk's operands from global memory into registers (zeros outside the chunk, the rows and
// the right-hand sides): thread (warp w, lane l) takes pair kk = 4 w + (l & 3) of the chunk,
// A rows m = 8 i + (l >> 2) and B rows n = 8 i + (l >> 2) of it
__device__ __forceinline__ void tc_load(const RowArgs<float2> &a, const TcWalk &k, const TcChunk &ch, TcLoad &L) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kq = lane & 3, rq = lane >> 2;
    const int kk = 4 * w + kq;
    const bool live = kk < ch.jn;
    // the pair's segment and column: kk steps on from the chunk's start
    int e = ch.e, j = ch.j0 + kk, we = k.w;
    if (live)
        while (j >= we) {
            j -= we;
            ++e;
            we = a.g_w[e];
        }
    const int64_t mo = live ? a.g_moff[e] : 0;
    const float *M = reinterpret_cast<const float *>((mo >= 0 ? a.M + mo : a.M2 + (-1 - mo)) + int64_t(j) * k.rec.ld +
                                                     k.rec.r0);
    const float *V = reinterpret_cast<const float *>(a.src32 + (live ? a.g_voff[e] + j : 0) * a.vs + ch.c0);
    const int nf = 2 * (a.b - ch.c0);  // floats of the right-hand sides of this pass
    const int nb = 2 * k.rec.R;
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        const int m = 8 * i + rq;
        L.a[i] = live && m < nf ? V[m] : 0.f;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int n = 8 * i + rq;
        L.b[i] = live && n < nb ? M[n] : 0.f;
    }
}

// the registers of a chunk, split into TF32 heads and tails, into stage `st`
__device__ __forceinline__ void tc_store(unsigned char *st, const TcLoad &L) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kq = lane & 3, rq = lane >> 2;
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        const int rest = 4 * i + w;
        const int k4 = rest & 3, mg = rest >> 2;
        const int tile = mg >> 4, kg = k4 >> 1;
        const int off = (mg & 15) * 256 + (k4 & 1) * 128 + rq * 16 + kq * 4;
        uint32_t hi, lo;
        split(L.a[i], hi, lo);
        *reinterpret_cast<uint32_t *>(st + a_off(0, tile, kg) + off) = hi;
        *reinterpret_cast<uint32_t *>(st + a_off(1, tile, kg) + off) = lo;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int rest = 4 * i + w;
        const int k4 = rest & 3, ng = rest >> 2;
        const int kg = k4 >> 1;
        const int off = ng * 256 + (k4 & 1) * 128 + rq * 16 + kq * 4;
        uint32_t hi, lo;
        split(L.b[i], hi, lo);
        *reinterpret_cast<uint32_t *>(st + b_off(0, kg) + off) = hi;
        *reinterpret_cast<uint32_t *>(st + b_off(1, kg) + off) = lo;
    }
}

// One output pass's results from tensor memory (or zero) into the arena or y. Thread (warp w, lane
// l) holds tile row m = 32 w + l: right-hand side c0 + 64 t + m / 2, part m & 1 of the vectors.
template <bool CONJ>
__device__ __forceinline__ void tc_epilogue(const RowArgs<float2> &a, uint32_t tmem, const WideOut &rec, int c0,
                                            bool zero) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int R = rec.R;
    const int npad = max(16, (2 * R + 15) & ~15);
    const bool scatter = a.y != nullptr;
    for (int t = 0; t < 2; ++t) {
        if (c0 + 64 * t >= a.b) break;
        const int c = c0 + 64 * t + ((32 * warp + lane) >> 1);
        for (int n0 = 0; n0 < npad; n0 += 16) {
            float v[16];
            if (zero) {
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] = 0.f;
            } else {
                tmem_ld16(tmem + (uint32_t(32 * warp) << 16) + uint32_t(128 * t + n0), v);
            }
            float p[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) p[i] = __shfl_xor_sync(0xffffffffu, v[i], 1);
            if ((lane & 1) || c >= a.b) continue;
            // v: part 0 (real) of the vectors, p: part 1 (imaginary)
#pragma unroll
            for (int rr = 0; rr < 8; ++rr) {
                const int r = n0 / 2 + rr;
                if (r >= R) break;
                float re, im;
                if (CONJ) {
                    re = v[2 * rr] + p[2 * rr + 1];
                    im = p[2 * rr] - v[2 * rr + 1];
                } else {
                    re = v[2 * rr] - p[2 * rr + 1];
                    im = v[2 * rr + 1] + p[2 * rr];
                }
                if (scatter) {
                    double2 *yp = a.y + a.perm[rec.out + r] + int64_t(c) * a.ldy;
                    double2 out = make_double2(a.alpha.x * re - a.alpha.y * im, a.alpha.x * im + a.alpha.y * re);
                    if (a.usebeta) {
                        const double2 yo = *yp;
                        out.x += a.beta.x * yo.x - a.beta.y * yo.y;
                        out.y += a.beta.x * yo.y + a.beta.y * yo.x;
                    }
                    *yp = out;
                } else {
                    float2 *d = a.dst32 + (rec.out + r) * a.vs + c;
                    float2 o = make_float2(re, im);
                    if (a.accumulate) {
                        const float2 old = *d;
                        o.x += old.x;
                        o.y += old.y;
                    }
                    *d = o;
                }
            }
        }
    }
}

template <bool CONJ>
__global__ void __launch_bounds__(TC_THREADS, 2) k_gather_tc(RowArgs<float2> a, const WideOut *outs, int count) {
    extern __shared__ __align__(1024) unsigned char tsm[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(tsm + 2 * TC_STAGE);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(tsm + 2 * TC_STAGE + 32);
    const int tid = threadIdx.x, warp = tid >> 5;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tslot)), "r"(256)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        bar_init(&bars[0], 1);
        bar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot;
    const uint32_t sbase = su32(tsm);

    TcWalk k;
    k.wi = blockIdx.x;
    tc_start_output(a, outs, count, k);
    TcChunk ch;
    bool have = tc_chunk(k, count, ch);
    TcLoad L;
    if (have && ch.jn > 0) tc_load(a, k, ch, L);
    // the previous chunk, whose pass may still need its epilogue
    bool pend = false, pend_zero = false;
    WideOut pend_rec{};
    int pend_c0 = 0, pend_stage = 0;
    uint32_t pend_parity = 0;
    int kc = 0;  // chunks committed so far (stage kc & 1, its use kc >> 1)
    bool stop = false;
    while (have && !stop) {
        // 1. the previous pass's results (its MMAs were committed one step ago; this chunk's loads
        //    are in flight meanwhile)
        if (pend) {
            if (!pend_zero && !bar_wait(&bars[pend_stage], pend_parity)) {
                stop = true;
                atomicExch(a.error, 2);
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (!stop) tc_epilogue<CONJ>(a, tmem, pend_rec, pend_c0, pend_zero);
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            pend = false;
        }
        if (ch.jn > 0) {
            const int s = kc & 1;
            // 2. the stage is free once the MMAs of two chunks ago are done
            if (kc >= 2 && !bar_wait(&bars[s], ((kc - 2) >> 1) & 1)) {
                stop = true;
                atomicExch(a.error, 2);
            }
            if (!stop) tc_store(tsm + s * TC_STAGE, L);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
        stop = __syncthreads_or(stop);
        if (stop) break;
        if (ch.jn > 0) {
            const int s = kc & 1;
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const int npad = max(16, (2 * k.rec.R + 15) & ~15);
                const uint32_t id = idesc_tf32(npad);
                const uint32_t st = sbase + uint32_t(s * TC_STAGE);
                const int tiles = a.b - ch.c0 > 64 ? 2 : 1;
                for (int kg = 0; kg < (ch.jn + 7) / 8; ++kg) {
                    const uint64_t bh = mdesc(st + b_off(0, kg), 128, 256);
                    const uint64_t bl = mdesc(st + b_off(1, kg), 128, 256);
                    for (int t = 0; t < tiles; ++t) {
                        const uint64_t ah = mdesc(st + a_off(0, t, kg), 128, 256);
                        const uint64_t al = mdesc(st + a_off(1, t, kg), 128, 256);
                        const uint32_t d = tmem + uint32_t(128 * t);
                        const bool acc = !(ch.first && kg == 0);
                        mma_tf32(d, ah, bh, id, acc);
                        mma_tf32(d, ah, bl, id, true);
                        mma_tf32(d, al, bh, id, true);
                    }
                }
                mma_commit(&bars[s]);
            }
        }
        // 3. remember the pass for its epilogue, step on, load the next chunk
        if (ch.last) {
            pend = true;
            pend_zero = ch.jn == 0;
            pend_rec = k.rec;
            pend_c0 = ch.c0;
            pend_stage = kc & 1;
            pend_parity = (kc >> 1) & 1;
        }
        if (ch.jn > 0) ++kc;
        tc_advance(a, outs, count, k);
        have = tc_chunk(k, count, ch);
        if (have && ch.jn > 0) tc_load(a, k, ch, L);
    }
    if (pend && !stop) {
        if (!pend_zero && !bar_wait(&bars[pend_stage], pend_parity)) {
            stop = true;
            atomicExch(a.error, 2);
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (!stop) tc_epilogue<CONJ>(a, tmem, pend_rec, pend_c0, pend_zero);
    }
    // every MMA is complete (each pass ended with a wait on its last commit) before the release
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256) : "memory");
    }
}

}  // namespace

bool gather_tc_fits(int maxrows) { return maxrows <= 64; }

size_t gather_tc_smem_bytes() { return size_t(TC_SMEM); }

void launch_gather_tc(const RowArgs<float2> &a, const WideOut *outs, int count, cudaStream_t s) {
    if (count <= 0) return;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = count < 2 * sms ? count : 2 * sms;
    if (a.conj) {
        cudaFuncSetAttribute(k_gather_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
        k_gather_tc<true><<<grid, TC_THREADS, TC_SMEM, s>>>(a, outs, count);
    } else {
        cudaFuncSetAttribute(k_gather_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
        k_gather_tc<false><<<grid, TC_THREADS, TC_SMEM, s>>>(a, outs, count);
    }
}

}  // namespace nca
