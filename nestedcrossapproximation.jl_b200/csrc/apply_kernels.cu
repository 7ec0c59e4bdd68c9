// Device kernel of the H^2 matrix-vector product (src/nca/aggregate.jl, couple.jl,
// disaggregate.jl and the near-field product of src/nca/petrovgalerkinnca.jl:431-589) for a
// block of b right-hand sides.
//
// Every stage is the same operation: for each output node o (one CTA),
//     out_o (R x b) = sum over segments  op(M_seg) (R x w_seg) * v_seg (w_seg x b)
// with every matrix block M_seg contiguous (column-major, leading dimension R) and every vector
// slice v_seg contiguous (rows of b right-hand sides, v[i * b + q]). The stores keep transposed
// copies where a product needs them, so each stage reads R x w tiles:
//   upward   xhat_p = X_p^T [xhat_c1; xhat_c2; ...] (leaf: the gathered x slice)   from XT
//   coupling yhat_t = sum_s S_ts xhat_s      (reverse: from the transposed couplings CT)
//   downward [yhat_c1; ...] += X_p yhat_p
//   leaves   y_t = X_t yhat_t + sum_s N_ts x_s (reverse: from the transposed near blocks NT),
//            scattered straight into the caller's layout.
//
// CTA = 8 consumer warps + 1 producer warp. The producer streams tiles through a 2-stage
// shared-memory ring with cp.async.bulk (bulk copies completing on a "full" mbarrier), filling
// each stage with columns of successive segments; the consumers release stages on an "empty"
// mbarrier. Tiles go through the FP64 tensor-core MMA (mma.m8n8k4.f64) with three real
// products per complex product (Re = ArBr - AiBi, Im = (Ar+Ai)(Br+Bi) - ArBr - AiBi); stored
// complex FP32 blocks are widened to FP64 as they are loaded, so both precisions accumulate in
// FP64 and FP32 storage halves the bytes streamed without changing the arithmetic. Output
// tiles of 8 rows x 8 right-hand sides are spread over the warps; when a node has fewer
// tiles than warps the columns are split between warps and summed in shared memory. Every
// wait is bounded: on timeout the CTA records an error, drains its copies (bounded) and
// returns. Every stage gathers (no atomics), so products are bitwise reproducible.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "apply_kernels.cuh"

namespace nca {

namespace {

constexpr int NCONS = 8;              // consumer warps
constexpr int NT = (NCONS + 1) * 32;  // + one producer warp
constexpr int NSTAGE = 2;
constexpr int STAGE_BYTES = 35328;  // one ring stage: w matrix columns, then w vector rows

// Shared-memory strides (in 16-byte elements) that are 2 mod 4: the four lanes of an MMA
// fragment row then hit four different bank groups.
__host__ __device__ __forceinline__ int conflict_free(int n) { return n + ((6 - n % 4) % 4); }
constexpr unsigned kWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx_only(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
    for (unsigned it = 0; it < kWaitLimit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// D = A (8x4, row) * B (4x8, col) + D on the FP64 tensor cores.
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// V: the vector element type (complex FP64; complex FP32 for the gathers of a complex-FP32
// coefficient arena)
template <typename S, typename V = double2>
struct Seg {
    const S *M;
    const V *v;
    int w;
};

// the gathers' input vectors and output rows in the arena's element type
template <typename V, typename S>
__device__ __forceinline__ const V *vec_src(const RowArgs<S> &a) {
    if constexpr (std::is_same<V, float2>::value) return a.src32;
    else return a.src;
}
template <typename V, typename S>
__device__ __forceinline__ V *vec_dst(const RowArgs<S> &a) {
    if constexpr (std::is_same<V, float2>::value) return a.dst32;
    else return a.dst;
}

template <typename S, int STAGE>
__device__ __forceinline__ int out_rows(const RowArgs<S> &a, int o) {
    if (STAGE == STAGE_UP) return a.rank[o];
    if (STAGE == STAGE_DOWN) return a.nrows[o];
    if (STAGE == STAGE_COUPLE) return a.rank_out[o];
    if (STAGE == STAGE_GATHER) return a.g_rows[o];
    return a.end[o] - a.begin[o];
}

template <typename S, int STAGE>
__device__ __forceinline__ int own_segment(const RowArgs<S> &a, int o) {
    return (STAGE == STAGE_LEAVES && a.X && a.rank[o] > 0) ? 1 : 0;
}

template <typename S, int STAGE>
__device__ __forceinline__ int nsegs(const RowArgs<S> &a, int o) {
    if (STAGE == STAGE_UP || STAGE == STAGE_DOWN) return 1;
    if (STAGE == STAGE_GATHER) return a.g_segptr[o + 1] - a.g_segptr[o];
    const int list = a.ptr ? a.ptr[o + 1] - a.ptr[o] : 0;
    return own_segment<S, STAGE>(a, o) + list;
}

template <typename S, int STAGE, typename V = double2>
__device__ __forceinline__ Seg<S, V> segment(const RowArgs<S> &a, int o, int k) {
    Seg<S, V> g;
    if constexpr (!std::is_same<V, double2>::value) {
        // complex-FP32 vectors: the block-sparse gathers only
        const int e = a.g_segptr[o] + k;
        const int64_t mo = a.g_moff[e];
        g.M = mo >= 0 ? a.M + mo : a.M2 + (-1 - mo);
        g.w = a.g_w[e];
        g.v = vec_src<V>(a) + a.g_voff[e] * a.vs;
        return g;
    } else if (STAGE == STAGE_UP) {
        g.M = a.M + a.moff[o];
        g.w = a.nrows[o];
        g.v = a.nchildren[o] == 0 ? a.src + int64_t(a.begin[o]) * a.vs : a.coef + a.cptr[a.firstchild[o]] * a.vs;
    } else if (STAGE == STAGE_DOWN) {
        g.M = a.M + a.moff[o];
        g.w = a.rank[o];
        g.v = a.coef + a.cptr[o] * a.vs;
    } else if (STAGE == STAGE_GATHER) {
        const int e = a.g_segptr[o] + k;
        const int64_t mo = a.g_moff[e];
        g.M = mo >= 0 ? a.M + mo : a.M2 + (-1 - mo);
        g.w = a.g_w[e];
        g.v = a.src + a.g_voff[e] * a.vs;
    } else if (STAGE == STAGE_COUPLE) {
        const int e = a.ptr[o] + k;
        const int other = a.other[e];
        g.M = a.M + a.moff[e];
        g.w = a.rank_in[other];
        g.v = a.src + a.cptr_in[other] * a.vs;
    } else {
        const int own = own_segment<S, STAGE>(a, o);
        if (k < own) {
            g.M = a.X + a.xoff[o];
            g.w = a.rank[o];
            g.v = a.coef + a.cptr[o] * a.vs;
        } else {
            const int e = a.ptr[o] + k - own;
            const int other = a.other[e];
            g.M = a.M + a.moff[e];
            g.w = a.o_end[other] - a.o_begin[other];
            g.v = a.src + int64_t(a.o_begin[other]) * a.vs;
        }
    }
    return g;
}

// Shared control block of one CTA.
struct Ctl {
    uint64_t full[NSTAGE];
    uint64_t empty[NSTAGE];
    int w[NSTAGE];
    int abort;
    int err;
};

// Per-warp accumulators: NRT row tiles x NTL column tiles of 8 x 8 outputs, the three real
// products of the 3M complex product per tile (c1 = Ar Br, c2 = Ai Bi, c3 = (Ar + s Ai)
// (Br + Bi) with s = -1 for the conjugate), in two independent sets (even / odd k-steps) when a
// warp holds a single tile. Both stored precisions accumulate in FP64.
template <int NRT, int NTL>
struct Acc {
    static constexpr int T = NRT * NTL;
    static constexpr int NSET = T <= 1 ? 2 : 1;
    double c1[NSET][T][2], c2[NSET][T][2], c3[NSET][T][2];
    __device__ void zero() {
#pragma unroll
        for (int p = 0; p < NSET; ++p)
#pragma unroll
            for (int u = 0; u < T; ++u)
#pragma unroll
                for (int h = 0; h < 2; ++h) c1[p][u][h] = c2[p][u][h] = c3[p][u][h] = 0.0;
    }
    // Re = c1 - s c2, Im = c3 - c1 - s c2 (s = +1: A B; s = -1: conj(A) B)
    __device__ double2 value(int u, int h, double sgn) const {
        double r1 = 0.0, r2 = 0.0, r3 = 0.0;
#pragma unroll
        for (int p = 0; p < NSET; ++p) {
            r1 += c1[p][u][h];
            r2 += c2[p][u][h];
            r3 += c3[p][u][h];
        }
        const double t = sgn * r2;
        return make_double2(r1 - t, r3 - r1 - t);
    }
};

__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2(v.x, v.y); }

// Output tiles of one consumer warp. The R x bc output is cut into row tiles of 8 rows; a warp
// owns whole row tiles (all NTL column tiles of 8 right-hand sides, so one A fragment serves
// them all): row tiles rt0, rt0 + 8, ... (nrt of them, at most NRT). When there are fewer row
// tiles than warps, the columns are split into kgroups interleaved groups of k-steps and the
// groups are summed at the end.
struct TileMap {
    int kgroups, mykg, rt0, nrt;
    int step = NCONS;  // row tiles between a warp's successive tiles
    // partial sums per output row: rows 0-31 and rows from 32 on (the same for every warp)
    int parts_lo = 1, parts_hi = 1;
    // one warp holding every tile of an R-row output (row tiles 0, 1, ...)
    __device__ void init_single(int R) {
        kgroups = 1;
        mykg = 0;
        rt0 = 0;
        nrt = (R + 7) >> 3;
        step = 1;
    }
    __device__ void init(int R, int warp) {
        const int MT = (R + 7) >> 3;
        if (MT == 5 || MT == 6) {
            // Four whole row tiles on warps 0-3 (one per SM sub-partition, warp w runs on
            // sub-partition w mod 4) and the other MT - 4 row tiles split by k-steps over warps
            // 4-7, so that every sub-partition's tensor pipe gets the same share (whole tiles on
            // warps 0-4 would give one sub-partition two tiles while the others have one).
            const int split = 4 / (MT - 4);
            if (warp < 4) {
                kgroups = 1;
                mykg = 0;
                rt0 = warp;
            } else {
                kgroups = split;
                mykg = (warp - 4) % split;
                rt0 = 4 + (warp - 4) / split;
            }
            nrt = 1;
            parts_lo = 1;
            parts_hi = split;
            return;
        }
        const int mt1 = MT > 0 ? MT : 1;
        kgroups = MT >= NCONS ? 1 : NCONS / mt1;
        mykg = kgroups > 1 ? warp / mt1 : 0;
        rt0 = kgroups > 1 ? warp % mt1 : warp;
        const bool busy = MT > 0 && (kgroups > 1 ? warp < MT * kgroups : warp < MT);
        nrt = !busy ? 0 : kgroups > 1 ? 1 : (MT - rt0 + NCONS - 1) / NCONS;
        parts_lo = parts_hi = kgroups;
    }
    __device__ int row(int j, int g) const { return (rt0 + j * step) * 8 + g; }
};

// One chunk (w columns, tile at smem offset 0, vectors at voff) of the consumer warp's tiles,
// on the FP64 tensor cores for both stored precisions (complex FP32 blocks are widened to FP64
// as their fragments are loaded). Operands of full k-steps are loaded without checks: A rows
// past R and B columns past bc only reach outputs that are never stored (each C row / column
// depends on its own A row / B column alone), so their addresses are clamped into the block.
// Only k-steps that cross the chunk end need zeros (a k past w would reach every output).
template <typename S, int NRT, int NTL, typename V = double2>
__device__ __forceinline__ void consume(Acc<NRT, NTL> &acc, const TileMap &tm, const unsigned char *tile, int w,
                                        int voff, int R, int ldm, int bc, int ldv, int g, int tq, double sgn) {
    const S *Ms = reinterpret_cast<const S *>(tile);
    const V *Vs = reinterpret_cast<const V *>(tile + voff);
    constexpr int NSET = Acc<NRT, NTL>::NSET;
    const int step = 4 * tm.kgroups;
    int ar[NRT], bcl[NTL];
#pragma unroll
    for (int j = 0; j < NRT; ++j) {
        const int r = tm.row(j, g);
        ar[j] = r < R ? r : R - 1;
    }
#pragma unroll
    for (int t = 0; t < NTL; ++t) bcl[t] = t * 8 + g < bc ? t * 8 + g : bc - 1;
    auto kstep = [&](int p, int kk, bool full) {
        double2 bv[NTL];
        double bs[NTL];
#pragma unroll
        for (int t = 0; t < NTL; ++t) {
            bv[t] = (full || kk < w) ? to_d2(Vs[kk * ldv + bcl[t]]) : make_double2(0.0, 0.0);
            bs[t] = bv[t].x + bv[t].y;
        }
#pragma unroll
        for (int j = 0; j < NRT; ++j) {
            if (NRT > 1 && j >= tm.nrt) break;
            const double2 av = (full || kk < w) ? to_d2(Ms[ar[j] + kk * ldm]) : make_double2(0.0, 0.0);
            const double as = fma(sgn, av.y, av.x);
#pragma unroll
            for (int t = 0; t < NTL; ++t) {
                const int u = j * NTL + t;
                dmma(acc.c1[p][u][0], acc.c1[p][u][1], av.x, bv[t].x);
                dmma(acc.c2[p][u][0], acc.c2[p][u][1], av.y, bv[t].y);
                dmma(acc.c3[p][u][0], acc.c3[p][u][1], as, bs[t]);
            }
        }
    };
    int k0 = tm.mykg * 4;
    // whole sets: every set of the group ends inside the chunk
    for (; k0 + (NSET - 1) * step + 4 <= w; k0 += NSET * step) {
#pragma unroll
        for (int p = 0; p < NSET; ++p) kstep(p, k0 + p * step + tq, true);
    }
    // the rest of the chunk: sets that start inside it, with zeros past w
#pragma unroll
    for (int p = 0; p < NSET; ++p) {
        const int kb = k0 + p * step;
        if (kb >= w) break;
        kstep(p, kb + tq, kb + 4 <= w);
    }
}

}  // namespace

int rows_capacity(int bc) {
    // at most 8 tiles of 8 x 8 per warp over 8 warps (R * ceil(bc / 8) <= 512); 4 padded complex
    // FP64 columns and their vector rows must fit one stage; the partial sums (R x bc) must fit
    // the ring
    const int ntl = (bc + 7) / 8;
    const int by_tiles = 512 / (ntl > 0 ? ntl : 1);
    const int by_tile_bytes = STAGE_BYTES / (4 * 16) - conflict_free(bc) - 3;
    const int by_ring = NSTAGE * STAGE_BYTES / (16 * (bc > 0 ? bc : 1));
    int cap = by_tiles < by_tile_bytes ? by_tiles : by_tile_bytes;
    return cap < by_ring ? cap : by_ring;
}

template <typename S, int STAGE, int NRT, int NTL, typename V = double2>
__device__ __forceinline__ void rows_body(const RowArgs<S> &a, const int32_t *nodes) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ Ctl ctl;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int o = nodes[blockIdx.x];
    if (STAGE == STAGE_UP && a.skip_leaves && a.nchildren[o] == 0) return;  // whole CTA, before any barrier
    const int R = out_rows<S, STAGE>(a, o);
    const int bc = a.bc;
    const int elem = int(sizeof(S));
    constexpr bool f64 = std::is_same<S, double2>::value;
    // FP64 blocks of 32 rows or more are copied column by column into padded shared-memory
    // columns (conflict-free A fragments); smaller blocks, whose many short columns would make
    // the producer the bottleneck, and FP32 tiles are copied in one piece per segment. Vector
    // rows keep the buffers' padded stride when a pass covers all right-hand sides.
    const bool percol = f64 && R >= 32;
    const int ldm = percol ? conflict_free(R) : R;
    const bool vwhole = bc == a.b;
    const int ldv = vwhole ? a.vs : conflict_free(bc);  // >= bc + 1 for odd bc
    constexpr int vel = int(sizeof(V));
    // columns per stage: matrix columns first, the vector rows at voff (16-byte aligned). Chunks
    // are whole groups of k-steps of 4, one per accumulator set, so interior FP32 chunks stay
    // 16-byte multiples.
    int wmax = STAGE_BYTES / (ldm * elem + ldv * vel);
    {
        constexpr int kq = 4 * Acc<NRT, NTL>::NSET;
        wmax = wmax >= kq ? wmax - wmax % kq : (wmax & ~3);
    }
    if (wmax < 4) wmax = 4;
    int voff = (wmax * ldm * elem + 15) & ~15;
    while (wmax > 4 && voff + wmax * ldv * vel > STAGE_BYTES) {
        wmax -= 4;
        voff = (wmax * ldm * elem + 15) & ~15;
    }

    if (tid == 0) {
        for (int s = 0; s < NSTAGE; ++s) {
            mbar_init(&ctl.full[s], 1);
            mbar_init(&ctl.empty[s], NCONS);
        }
        ctl.abort = 0;
        ctl.err = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const int g = lane >> 2, tq = lane & 3;
    volatile int *abort_flag = &ctl.abort;
    Acc<NRT, NTL> acc;
    acc.zero();
    TileMap tm;
    tm.init(R, warp < NCONS ? warp : 0);
    const double sgn = a.conj ? -1.0 : 1.0;

    if (warp == NCONS) {
        // ---------------- producer warp ----------------
        if (lane == 0) {
            const int nseg = nsegs<S, STAGE>(a, o);
            int k = 0, c0 = 0;
            // the next segment's descriptor is loaded one segment ahead, so the dependent index
            // loads (CSR entry -> partner node -> its range) overlap the current segment's copies
            Seg<S, V> gs, gnext;
            gs.w = 0;
            gnext.w = 0;
            if (nseg > 0) gs = segment<S, STAGE, V>(a, o, 0);
            if (nseg > 1) gnext = segment<S, STAGE, V>(a, o, 1);
            for (int chunk = 0;; ++chunk) {
                const int s = chunk % NSTAGE;
                if (chunk >= NSTAGE && !mbar_wait_bounded(&ctl.empty[s], ((chunk / NSTAGE) - 1) & 1)) {
                    *abort_flag = 1;
                    break;
                }
                if (*abort_flag) break;
                unsigned char *tile = smem + s * STAGE_BYTES;
                // The stage is filled with columns of successive segments: complex FP64 pieces
                // (and FP32 pieces of an even number of rows) are whole 16-byte multiples, so
                // they pack at any column; odd-row FP32 tiles are one piece each.
                int filled = 0;
                while (filled < wmax) {
                    while (k < nseg && c0 >= gs.w) {
                        ++k;
                        c0 = 0;
                        gs = gnext;
                        if (k + 1 < nseg) gnext = segment<S, STAGE, V>(a, o, k + 1);
                    }
                    if (k >= nseg) break;
                    int w = gs.w - c0;
                    if (w > wmax - filled) w = wmax - filled;
                    const S *msrc = gs.M + int64_t(c0) * R;
                    const V *vsrc = gs.v + int64_t(c0) * a.vs + a.q0;
                    c0 += w;
                    if (((reinterpret_cast<uintptr_t>(msrc) | reinterpret_cast<uintptr_t>(vsrc)) & 15u) != 0) {
                        ctl.err = 1;  // never issue an unaligned bulk copy: skip this piece
                        continue;
                    }
                    // a row of bc complex-FP32 values is rounded up to 16 bytes (an odd bc only
                    // occurs in the last pass of an odd b, whose rows have a padding slot)
                    const uint32_t vrow = (uint32_t(bc) * uint32_t(vel) + 15u) & ~15u;
                    const uint32_t vbytes = vwhole ? uint32_t(w) * uint32_t(a.vs) * uint32_t(vel) : vrow * uint32_t(w);
                    unsigned char *mdst = tile + filled * ldm * elem;
                    unsigned char *vdst = tile + voff + filled * ldv * vel;
                    if (percol) {
                        const uint32_t col = uint32_t(R) * 16u;
                        mbar_expect_tx_only(&ctl.full[s], col * uint32_t(w) + vbytes);
                        for (int j = 0; j < w; ++j)
                            bulk_g2s(mdst + j * ldm * 16, msrc + int64_t(j) * R, col, &ctl.full[s]);
                    } else {
                        const uint32_t mbytes = (uint32_t(R) * uint32_t(w) * uint32_t(elem) + 15u) & ~15u;
                        mbar_expect_tx_only(&ctl.full[s], mbytes + vbytes);
                        if (mbytes) bulk_g2s(mdst, msrc, mbytes, &ctl.full[s]);
                    }
                    if (vwhole) {
                        bulk_g2s(vdst, vsrc, vbytes, &ctl.full[s]);
                    } else {
                        for (int j = 0; j < w; ++j)
                            bulk_g2s(vdst + j * ldv * vel, vsrc + int64_t(j) * a.vs, vrow, &ctl.full[s]);
                    }
                    filled += w;
                    if (!f64 && (R & 1)) break;  // odd-row FP32 pieces may end off a 16-byte boundary
                }
                if (filled == 0 && k >= nseg) {
                    ctl.w[s] = -1;
                    mbar_arrive(&ctl.full[s]);
                    break;
                }
                ctl.w[s] = filled;
                mbar_arrive(&ctl.full[s]);
            }
        }
        __syncwarp();
    } else {
        // ---------------- consumer warps ----------------
        for (int chunk = 0;; ++chunk) {
            const int s = chunk % NSTAGE;
            if (!mbar_wait_bounded(&ctl.full[s], (chunk / NSTAGE) & 1)) {
                *abort_flag = 1;
                break;
            }
            const int w = ctl.w[s];
            if (w < 0 || *abort_flag) break;
            if (tm.nrt > 0)
                consume<S, NRT, NTL, V>(acc, tm, smem + s * STAGE_BYTES, w, voff, R, ldm, bc, ldv, g, tq, sgn);
            __syncwarp();
            if (lane == 0) mbar_arrive(&ctl.empty[s]);
        }
    }
    __syncthreads();  // every role is done with the ring
    const bool aborted = *abort_flag != 0;
    double2 *red = reinterpret_cast<double2 *>(smem);
    if (!aborted && warp < NCONS) {
#pragma unroll
        for (int j = 0; j < NRT; ++j) {
            if (j >= tm.nrt) break;
            const int row = tm.row(j, g);  // C fragment rows equal the A fragment rows (g)
            if (row >= R) continue;
#pragma unroll
            for (int t = 0; t < NTL; ++t)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int col = t * 8 + 2 * tq + h;
                    if (col < bc) red[(tm.mykg * R + row) * bc + col] = acc.value(j * NTL + t, h, sgn);
                }
        }
    }
    __syncthreads();  // partial sums visible
    if (aborted) {
        // a wait gave up: wait (bounded) for copies that may still land in the ring, then leave
        if (tid == 0) {
            for (int s = 0; s < NSTAGE; ++s) {
                mbar_wait_bounded(&ctl.full[s], 0);
                mbar_wait_bounded(&ctl.full[s], 1);
            }
            atomicCAS(a.error, 0, 2);
        }
        return;
    }
    if (tid == 0 && ctl.err) atomicCAS(a.error, 0, ctl.err);
    const bool scatter = STAGE == STAGE_LEAVES || (STAGE == STAGE_GATHER && a.y != nullptr);
    for (int e = tid; e < R * bc; e += NT) {
        // coefficients: right-hand sides fastest (contiguous rows); y: rows fastest (the caller's columns)
        const int i = scatter ? e % R : e / bc;
        const int qq = scatter ? e / R : e % bc;
        double2 v = red[i * bc + qq];
        const int parts = i < 32 ? tm.parts_lo : tm.parts_hi;
        for (int kg = 1; kg < parts; ++kg) {
            const double2 p = red[(kg * R + i) * bc + qq];
            v.x += p.x;
            v.y += p.y;
        }
        const int col = a.q0 + qq;
        if constexpr (!std::is_same<V, double2>::value) {
            if (!scatter) {  // complex-FP32 arena rows
                V *d = vec_dst<V>(a) + (a.g_out[o] + i) * a.vs + col;
                if (a.accumulate) {
                    const V old = *d;
                    v = make_double2(double(old.x) + v.x, double(old.y) + v.y);
                }
                *d = V{float(v.x), float(v.y)};
                continue;
            }
        }
        if (STAGE == STAGE_UP || STAGE == STAGE_COUPLE || (STAGE == STAGE_GATHER && !scatter)) {
            double2 *d = STAGE == STAGE_UP       ? (a.coef_out ? a.coef_out : a.coef) + (a.cptr[o] + i) * a.vs + col
                         : STAGE == STAGE_COUPLE ? a.dst + (a.cptr_out[o] + i) * a.vs + col
                                                 : a.dst + (a.g_out[o] + i) * a.vs + col;
            if (a.accumulate) {
                const double2 old = *d;
                v = make_double2(old.x + v.x, old.y + v.y);
            }
            *d = v;
        } else if (STAGE == STAGE_DOWN) {
            double2 *d = (a.coef_out ? a.coef_out : a.coef) + (a.cptr[a.firstchild[o]] + i) * a.vs + col;
            const double2 old = *d;
            *d = make_double2(old.x + v.x, old.y + v.y);
        } else {
            const int64_t pos = STAGE == STAGE_GATHER ? a.g_out[o] + i : int64_t(a.begin[o]) + i;
            double2 *yp = a.y + a.perm[pos] + int64_t(col) * a.ldy;
            double2 out = make_double2(a.alpha.x * v.x - a.alpha.y * v.y, a.alpha.x * v.y + a.alpha.y * v.x);
            if (a.usebeta) {
                const double2 yo = *yp;
                out.x += a.beta.x * yo.x - a.beta.y * yo.y;
                out.y += a.beta.x * yo.y + a.beta.y * yo.x;
            }
            *yp = out;
        }
    }
}

// One kernel symbol per stage (the profiler and the launch list name them apart); a consumer
// warp keeps NRT row tiles x NTL column tiles of 8 x 8 outputs in registers.
#define NCA_ROWS_KERNEL(NAME, STAGE_ID)                                                           \
    template <typename S, int NRT, int NTL>                                                       \
    __global__ void __launch_bounds__(NT, NRT * NTL <= 2 ? 3 : 1) NAME(RowArgs<S> a, const int32_t *nodes) { \
        rows_body<S, STAGE_ID, NRT, NTL>(a, nodes);                                               \
    }
NCA_ROWS_KERNEL(k_rows_up, STAGE_UP)
NCA_ROWS_KERNEL(k_rows_couple, STAGE_COUPLE)
NCA_ROWS_KERNEL(k_rows_down, STAGE_DOWN)
NCA_ROWS_KERNEL(k_rows_leaves, STAGE_LEAVES)
#undef NCA_ROWS_KERNEL
template <typename S, int NRT, int NTL, typename V>
__global__ void __launch_bounds__(NT, NRT * NTL <= 2 ? 3 : 1) k_rows_gather(RowArgs<S> a, const int32_t *nodes) {
    rows_body<S, STAGE_GATHER, NRT, NTL, V>(a, nodes);
}

size_t rows_smem_bytes() { return size_t(NSTAGE) * STAGE_BYTES; }

__global__ void k_gather(const double2 *x, int64_t ldx, const int32_t *perm, int64_t n, int b, int vs,
                         double2 *xt) {
    const int64_t total = n * b;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
         e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t i = e / b;
        const int q = int(e % b);
        xt[i * vs + q] = x[perm[i] + q * ldx];
    }
}

__global__ void k_gather_to_f32(const double2 *x, int64_t ldx, const int32_t *perm, int64_t n, int b, int vs,
                                float2 *xt) {
    const int64_t total = n * b;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
         e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t i = e / b;
        const int q = int(e % b);
        const double2 v = x[perm[i] + q * ldx];
        xt[i * vs + q] = make_float2(float(v.x), float(v.y));
    }
}

int vector_stride(int b) { return conflict_free(b); }

namespace {
// One product launch; with a nonzero priority as a per-launch attribute, which a stream capture
// keeps in the graph (a graph does not carry its streams' priorities).
template <typename S, typename K>
void launch_one(K kern, const RowArgs<S> &a, const int32_t *nodes, int count, cudaStream_t s, size_t sm, int priority) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
    if (priority == 0) {
        kern<<<count, NT, sm, s>>>(a, nodes);
        return;
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(count);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = sm;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributePriority;
    at[0].val.priority = priority;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, a, nodes);
}

template <typename S, int NRT, int NTL>
void launch_tiles(const RowArgs<S> &a, const int32_t *nodes, int count, cudaStream_t s, size_t sm, int priority) {
    switch (a.stage) {
    case STAGE_UP:
        launch_one<S>(k_rows_up<S, NRT, NTL>, a, nodes, count, s, sm, priority);
        break;
    case STAGE_COUPLE:
        launch_one<S>(k_rows_couple<S, NRT, NTL>, a, nodes, count, s, sm, priority);
        break;
    case STAGE_DOWN:
        launch_one<S>(k_rows_down<S, NRT, NTL>, a, nodes, count, s, sm, priority);
        break;
    case STAGE_GATHER:
        launch_one<S>(k_rows_gather<S, NRT, NTL, double2>, a, nodes, count, s, sm, priority);
        break;
    default:
        launch_one<S>(k_rows_leaves<S, NRT, NTL>, a, nodes, count, s, sm, priority);
    }
}

// Row tiles per warp for the largest block of the launch: 1, 2, 4 or (one column tile only) 8;
// rows_capacity keeps R * ceil(bc / 8) <= 512, so the tiles of a warp never exceed 8.
template <typename S, int NTL>
void launch_ntl(const RowArgs<S> &a, const int32_t *nodes, int count, cudaStream_t s, size_t sm, int priority) {
    const int MT = (a.maxrows + 7) / 8;
    const int nrt = (MT + NCONS - 1) / NCONS;
    if (nrt <= 1)
        launch_tiles<S, 1, NTL>(a, nodes, count, s, sm, priority);
    else if (nrt <= 2)
        launch_tiles<S, 2, NTL>(a, nodes, count, s, sm, priority);
    else if (nrt <= 4 || NTL == 2)
        launch_tiles<S, 4, NTL>(a, nodes, count, s, sm, priority);
    else
        launch_tiles<S, (NTL == 1 ? 8 : 4), NTL>(a, nodes, count, s, sm, priority);
}
}  // namespace

template <typename S>
void launch_rows(const RowArgs<S> &a, const int32_t *nodes, int count, cudaStream_t s, size_t smem_bytes,
                 int priority) {
    if (count <= 0) return;
    const size_t sm = smem_bytes ? smem_bytes : rows_smem_bytes();
    if (a.bc > 8)
        launch_ntl<S, 2>(a, nodes, count, s, sm, priority);
    else
        launch_ntl<S, 1>(a, nodes, count, s, sm, priority);
}

template void launch_rows<double2>(const RowArgs<double2> &, const int32_t *, int, cudaStream_t, size_t, int);
template void launch_rows<float2>(const RowArgs<float2> &, const int32_t *, int, cudaStream_t, size_t, int);


namespace {
__device__ __forceinline__ double2 widen(double2 v) { return v; }
__device__ __forceinline__ double2 widen(float2 v) { return make_double2(v.x, v.y); }
template <typename T>
__device__ __forceinline__ T narrow(double2 v) {
    if constexpr (std::is_same<T, float2>::value) return make_float2(float(v.x), float(v.y));
    else return v;
}

// One warp per output of R <= 64 rows. RG = lanes per row group (a power of two >= min(R, 32));
// the 32 / RG column groups of the warp take the segment columns round robin and are summed by
// shuffles at the end; with R > 32 every lane keeps two rows. QB right-hand sides per pass; U
// columns per step, their loads issued together so that one memory round trip serves U columns.
template <typename S, int QB, int U, typename VT>
__global__ void __launch_bounds__(256) k_gather_small(RowArgs<S> a, const int32_t *nodes, int count) {
    const int lane = threadIdx.x & 31;
    const int wid = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (wid >= count) return;
    const int o = nodes[wid];
    const int R = a.g_rows[o];
    int RG = 32;
    while (RG > 1 && RG / 2 >= R) RG >>= 1;
    const int CG = 32 / RG;
    const int r0 = lane % RG, cg = lane / RG;
    const bool two = R > 32;
    const int e0 = a.g_segptr[o], e1 = a.g_segptr[o + 1];
    const double sg = a.conj ? -1.0 : 1.0;
    const bool scatter = a.y != nullptr;
    for (int qb = 0; qb < a.bc; qb += QB) {
        const int nq = a.bc - qb < QB ? a.bc - qb : QB;
        double2 acc0[QB], acc1[QB];
#pragma unroll
        for (int q = 0; q < QB; ++q) acc0[q] = acc1[q] = make_double2(0.0, 0.0);
        for (int e = e0; e < e1; ++e) {
            const int64_t mo = a.g_moff[e];
            const S *M = mo >= 0 ? a.M + mo : a.M2 + (-1 - mo);
            const int w = a.g_w[e];
            const VT *V = vec_src<VT>(a) + a.g_voff[e] * a.vs + a.q0 + qb;
            for (int j0 = cg; j0 < w; j0 += U * CG) {
                double2 m0[U], m1[U], x[U][QB];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int j = j0 + u * CG;
                    const bool in = j < w;
                    m0[u] = in && r0 < R ? widen(M[r0 + int64_t(j) * R]) : make_double2(0.0, 0.0);
                    m1[u] = in && two && r0 + 32 < R ? widen(M[r0 + 32 + int64_t(j) * R]) : make_double2(0.0, 0.0);
#pragma unroll
                    for (int q = 0; q < QB; ++q)
                        x[u][q] = in && q < nq ? widen(V[int64_t(j) * a.vs + q]) : make_double2(0.0, 0.0);
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    m0[u].y *= sg;
                    m1[u].y *= sg;
#pragma unroll
                    for (int q = 0; q < QB; ++q) {
                        const double2 xv = x[u][q];
                        acc0[q].x = fma(m0[u].x, xv.x, fma(-m0[u].y, xv.y, acc0[q].x));
                        acc0[q].y = fma(m0[u].x, xv.y, fma(m0[u].y, xv.x, acc0[q].y));
                        if (two) {
                            acc1[q].x = fma(m1[u].x, xv.x, fma(-m1[u].y, xv.y, acc1[q].x));
                            acc1[q].y = fma(m1[u].x, xv.y, fma(m1[u].y, xv.x, acc1[q].y));
                        }
                    }
                }
            }
        }
        // sum the column groups (lane bits above the row group)
        for (int off = RG; off < 32; off <<= 1) {
#pragma unroll
            for (int q = 0; q < QB; ++q) {
                acc0[q].x += __shfl_xor_sync(0xffffffffu, acc0[q].x, off);
                acc0[q].y += __shfl_xor_sync(0xffffffffu, acc0[q].y, off);
                if (two) {
                    acc1[q].x += __shfl_xor_sync(0xffffffffu, acc1[q].x, off);
                    acc1[q].y += __shfl_xor_sync(0xffffffffu, acc1[q].y, off);
                }
            }
        }
        if (cg != 0) continue;
        for (int h = 0; h < (two ? 2 : 1); ++h) {
            const int i = r0 + 32 * h;
            if (i >= R) continue;
#pragma unroll
            for (int q = 0; q < QB; ++q) {
                if (q >= nq) break;
                double2 v = h ? acc1[q] : acc0[q];
                const int col = a.q0 + qb + q;
                if (scatter) {
                    double2 *yp = a.y + a.perm[a.g_out[o] + i] + int64_t(col) * a.ldy;
                    double2 out = make_double2(a.alpha.x * v.x - a.alpha.y * v.y, a.alpha.x * v.y + a.alpha.y * v.x);
                    if (a.usebeta) {
                        const double2 yo = *yp;
                        out.x += a.beta.x * yo.x - a.beta.y * yo.y;
                        out.y += a.beta.x * yo.y + a.beta.y * yo.x;
                    }
                    *yp = out;
                } else {
                    VT *d = vec_dst<VT>(a) + (a.g_out[o] + i) * a.vs + col;
                    if (a.accumulate) {
                        const double2 old = widen(*d);
                        v = make_double2(old.x + v.x, old.y + v.y);
                    }
                    *d = narrow<VT>(v);
                }
            }
        }
    }
}
}  // namespace

template <typename S, typename VT>
void launch_gather_small(const RowArgs<S> &a, const int32_t *nodes, int count, cudaStream_t s) {
    if (count <= 0) return;
    const int grid = (count + 7) / 8;
    if (a.bc <= 1)
        k_gather_small<S, 1, 8, VT><<<grid, 256, 0, s>>>(a, nodes, count);
    else if (a.bc <= 4)
        k_gather_small<S, 4, 2, VT><<<grid, 256, 0, s>>>(a, nodes, count);
    else
        k_gather_small<S, 8, 1, VT><<<grid, 256, 0, s>>>(a, nodes, count);
}

template void launch_gather_small<double2, double2>(const RowArgs<double2> &, const int32_t *, int, cudaStream_t);
template void launch_gather_small<float2, double2>(const RowArgs<float2> &, const int32_t *, int, cudaStream_t);
template void launch_gather_small<float2, float2>(const RowArgs<float2> &, const int32_t *, int, cudaStream_t);

namespace {
// STAGE_GATHER over complex-FP32 stores and a complex-FP32 arena, every right-hand side of the
// product in one launch, for outputs of at most NR rows.
//
// One warp takes a grid-stride sequence of outputs; lane l holds columns c0 + 2 l and c0 + 2 l + 1
// of every output row in FP32 registers (passes c0 = 0, 64, ...). An output's segments are one
// sequence of W = sum w_e (block column, vector row) pairs, cut into chunks of WIDE_J pairs; the
// warp streams the chunks of all its (output, pass) steps through a WIDE_SLOTS-slot shared-memory
// ring filled by asynchronous copies, WIDE_SLOTS - 1 chunks ahead of the one being multiplied (a
// chunk of the next output is in flight while the current one finishes). A chunk holds the R
// entries of each block column (leading dimension NR, so one 16-byte shared load broadcasts two
// rows' entries to every lane) and each lane's two columns of each vector row. The multiply skips
// the row pairs at and beyond R. Complex FP32 FMA with FP32 accumulation.
constexpr int WIDE_WARPS = 4;  // warps (independent output sequences) per CTA
constexpr int WIDE_J = 8;      // (block column, vector row) pairs per chunk
constexpr int WIDE_SLOTS = 3;  // chunks per warp's ring

template <int NR, int CPL>
struct WideShape {
    static constexpr int mslot = NR * WIDE_J;        // float2 entries of a chunk's block columns
    static constexpr int vslot = WIDE_J * 32 * CPL;  // float2 entries of a chunk's vector rows
    static constexpr int slot = mslot + vslot;
    static constexpr size_t smem = size_t(WIDE_WARPS) * WIDE_SLOTS * slot * sizeof(float2);
};

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

__device__ __forceinline__ WideOut wide_record(const WideOut *outs, int i, int count) {
    WideOut o{0, 0, 0, 0, 0, 0, 0};
    if (i < count) {
        const int4 *q = reinterpret_cast<const int4 *>(outs + i);
        const int4 u = __ldg(q), v = __ldg(q + 1);
        o.R = u.x;
        o.W = u.y;
        o.e0 = u.z;
        o.e1 = u.w;
        o.out = int64_t((uint64_t(uint32_t(v.y)) << 32) | uint32_t(v.x));
        o.ld = v.z;
        o.r0 = v.w;
    }
    return o;
}

// lane l's share of a window of 32 segments starting at base: segment base + l
struct WideSeg {
    int w;
    int64_t moff, voff;
};
__device__ __forceinline__ WideSeg wide_segs(const RowArgs<float2> &a, int base, int e1, int lane) {
    WideSeg g{0, 0, 0};
    const int e = base + lane;
    if (e < e1) {
        g.w = __ldg(a.g_w + e);
        g.moff = __ldg(reinterpret_cast<const long long *>(a.g_moff) + e);
        g.voff = __ldg(reinterpret_cast<const long long *>(a.g_voff) + e);
    }
    return g;
}

template <int NR, int CPL, bool CONJ>
__global__ void __launch_bounds__(WIDE_WARPS * 32, CPL == 4 ? 2 : NR <= 8 ? 4 : NR <= 20 ? 3 : 2)
    k_gather_wide(RowArgs<float2> a, const WideOut *outs, int count) {
    using Shape = WideShape<NR, CPL>;
    extern __shared__ __align__(16) float2 wsm[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    float2 *ring = wsm + size_t(wib) * WIDE_SLOTS * Shape::slot;
    const int nw = int((int64_t(gridDim.x) * blockDim.x) >> 5);
    const int first = int((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    const bool scatter = a.y != nullptr;
    // ---- producer: walks the warp's outputs (records prefetched two ahead, segment windows one
    // ahead), their passes and their (block column, vector row) pairs, WIDE_J pairs per chunk
    int pwi = first;
    WideOut pc = wide_record(outs, first, count), pn = wide_record(outs, first + nw, count),
            p2 = wide_record(outs, first + 2 * nw, count);
    WideSeg gc = wide_segs(a, pc.e0, pc.e1, lane), gn = wide_segs(a, pn.e0, pn.e1, lane);
    int sb = pc.e0;           // first segment of the window in gc
    int pc0 = 0, pe = pc.e0, pj = 0, pt = 0;
    // the current segment's width, block and vector row (uniform)
    auto seg_at = [&](int e, int &w, const float2 *&M, int64_t &vb) {
        if (e < sb || e - sb >= 32) {
            sb = e;
            gc = wide_segs(a, sb, pc.e1, lane);
        }
        const int l = e - sb;
        w = __shfl_sync(0xffffffffu, gc.w, l);
        const long long mo = __shfl_sync(0xffffffffu, (long long)gc.moff, l);
        vb = __shfl_sync(0xffffffffu, (long long)gc.voff, l);
        M = mo >= 0 ? a.M + mo : a.M2 + (-1 - mo);
    };
    int pw = 0;
    const float2 *pM = nullptr;
    int64_t pvb = 0;
    if (pwi < count && pc.W > 0) seg_at(pe, pw, pM, pvb);
    auto issue = [&](int q) {
        // skip the (output, pass) steps whose pairs are all issued
        while (pwi < count && pt >= pc.W) {
            pc0 += 32 * CPL;
            pt = 0;
            pj = 0;
            pe = pc.e0;
            if (pc0 >= a.b || pc.W == 0) {
                pwi += nw;
                pc = pn;
                gc = gn;
                sb = pc.e0;
                pn = p2;
                gn = wide_segs(a, pn.e0, pn.e1, lane);
                p2 = wide_record(outs, pwi + 2 * nw, count);
                pc0 = 0;
                pe = pc.e0;
            }
            if (pwi < count && pc.W > 0) seg_at(pe, pw, pM, pvb);
        }
        if (pwi < count) {
            const int jn = min(WIDE_J, pc.W - pt);
            float2 *Ms = ring + q * Shape::slot;
            float2 *Vs = Ms + Shape::mslot;
            const int col = pc0 + CPL * lane;
            const int ncol = col < a.b ? min(CPL, a.b - col) : 0;
            const int R = pc.R;
            for (int jj = 0; jj < jn; ++jj) {
                while (pj >= pw) {
                    ++pe;
                    pj = 0;
                    seg_at(pe, pw, pM, pvb);
                }
                if (lane < R) cp_async8(Ms + jj * NR + lane, pM + int64_t(pj) * pc.ld + pc.r0 + lane);
                const float2 *v = a.src32 + (pvb + pj) * a.vs + col;
                float2 *d = Vs + (jj * 32 + lane) * CPL;
                if (ncol == CPL) {
#pragma unroll
                    for (int c = 0; c < CPL; c += 2) cp_async16(d + c, v + c);
                } else {
                    for (int c = 0; c < ncol; ++c) cp_async8(d + c, v + c);
                }
                ++pj;
            }
            pt += jn;
        }
        cp_async_commit();
    };
#pragma unroll
    for (int k = 0; k + 1 < WIDE_SLOTS; ++k) issue(k);
    // ---- consumer: the same walk, one chunk at a time out of the ring
    int qc = 0, qp = WIDE_SLOTS - 1;
    WideOut cc = wide_record(outs, first, count), cn = wide_record(outs, first + nw, count);
    for (int wi = first; wi < count; wi += nw) {
        const int R = cc.R, W = cc.W;
        const int64_t gout = cc.out;
        cc = cn;
        cn = wide_record(outs, wi + 2 * nw, count);
        for (int c0 = 0; c0 < a.b; c0 += 32 * CPL) {
            const int col = c0 + CPL * lane;
            const int ncol = col < a.b ? min(CPL, a.b - col) : 0;
            float2 acc[NR][CPL];
#pragma unroll
            for (int r = 0; r < NR; ++r)
#pragma unroll
                for (int c = 0; c < CPL; ++c) acc[r][c] = make_float2(0.f, 0.f);
            for (int t = 0; t < W; t += WIDE_J) {
                const int jn = min(WIDE_J, W - t);
                issue(qp);
                qp = qp + 1 == WIDE_SLOTS ? 0 : qp + 1;
                cp_async_wait<WIDE_SLOTS - 1>();
                __syncwarp();
                const float2 *Ms = ring + qc * Shape::slot;
                // lane's CPL columns of pair jj: float4 jj * 16 CPL + lane CPL / 2 + c
                const float4 *Vs = reinterpret_cast<const float4 *>(Ms + Shape::mslot) + lane * (CPL / 2);
                float4 xn[CPL / 2];
#pragma unroll
                for (int c = 0; c < CPL / 2; ++c) xn[c] = Vs[c];
#pragma unroll 1
                for (int jj = 0; jj < jn; ++jj) {
                    // this pair's vector columns; the next pair's loads issued before the FMAs
                    float4 x[CPL / 2];
#pragma unroll
                    for (int c = 0; c < CPL / 2; ++c) {
                        x[c] = xn[c];
                        xn[c] = Vs[min(jj + 1, WIDE_J - 1) * 16 * CPL + c];
                    }
                    const float4 *Mj = reinterpret_cast<const float4 *>(Ms + jj * NR);
#pragma unroll
                    for (int r2 = 0; r2 < NR / 2; ++r2) {
                        const float4 m2 = Mj[r2];
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const float mx = h ? m2.z : m2.x, my = CONJ ? -(h ? m2.w : m2.y) : (h ? m2.w : m2.y);
#pragma unroll
                            for (int c = 0; c < CPL / 2; ++c) {
                                float2 &p0 = acc[2 * r2 + h][2 * c], &p1 = acc[2 * r2 + h][2 * c + 1];
                                p0.x = fmaf(mx, x[c].x, fmaf(-my, x[c].y, p0.x));
                                p0.y = fmaf(mx, x[c].y, fmaf(my, x[c].x, p0.y));
                                p1.x = fmaf(mx, x[c].z, fmaf(-my, x[c].w, p1.x));
                                p1.y = fmaf(mx, x[c].w, fmaf(my, x[c].z, p1.y));
                            }
                        }
                    }
                }
                __syncwarp();
                qc = qc + 1 == WIDE_SLOTS ? 0 : qc + 1;
            }
            if (ncol == 0) continue;
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                if (r >= R) break;
                if (scatter) {
                    const int64_t yr = a.perm[gout + r];
#pragma unroll
                    for (int c = 0; c < CPL; ++c) {
                        if (c >= ncol) break;
                        const float2 v = acc[r][c];
                        double2 *yp = a.y + yr + int64_t(col + c) * a.ldy;
                        double2 out = make_double2(a.alpha.x * v.x - a.alpha.y * v.y, a.alpha.x * v.y + a.alpha.y * v.x);
                        if (a.usebeta) {
                            const double2 yo = *yp;
                            out.x += a.beta.x * yo.x - a.beta.y * yo.y;
                            out.y += a.beta.x * yo.y + a.beta.y * yo.x;
                        }
                        *yp = out;
                    }
                } else {
                    float2 *d = a.dst32 + (gout + r) * a.vs + col;
#pragma unroll
                    for (int c = 0; c < CPL; ++c) {
                        if (c >= ncol) break;
                        float2 v = acc[r][c];
                        if (a.accumulate) {
                            v.x += d[c].x;
                            v.y += d[c].y;
                        }
                        d[c] = v;
                    }
                }
            }
        }
    }
    cp_async_wait<0>();
}

template <int NR, int CPL, bool CONJ>
void wide_launch(const RowArgs<float2> &a, const WideOut *outs, int count, cudaStream_t s, int sms) {
    const size_t sm = WideShape<NR, CPL>::smem;
    auto kern = k_gather_wide<NR, CPL, CONJ>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WIDE_WARPS * 32, sm);
    const int need = (count + WIDE_WARPS - 1) / WIDE_WARPS;
    const int cap = sms * (per_sm > 0 ? per_sm : 1);
    kern<<<need < cap ? need : cap, WIDE_WARPS * 32, sm, s>>>(a, outs, count);
}

// four columns per lane (one pass over up to 128 right-hand sides) for tiles of up to 12 rows when
// the block has more than 64 columns; two otherwise
template <int NR>
void wide_launch(const RowArgs<float2> &a, const WideOut *outs, int count, cudaStream_t s, int sms) {
    if constexpr (NR <= 12) {
        if (a.b > 64) {
            if (a.conj)
                wide_launch<NR, 4, true>(a, outs, count, s, sms);
            else
                wide_launch<NR, 4, false>(a, outs, count, s, sms);
            return;
        }
    }
    if (a.conj)
        wide_launch<NR, 2, true>(a, outs, count, s, sms);
    else
        wide_launch<NR, 2, false>(a, outs, count, s, sms);
}
}  // namespace

bool gather_wide_fits(int maxrows) { return maxrows <= 32; }

int wide_rows_class(int R) {
    if (R <= 24) return R <= 2 ? 2 : R + (R & 1);
    return R <= 28 ? 28 : 32;
}

void launch_gather_wide(const RowArgs<float2> &a, const WideOut *outs, int count, int nr, cudaStream_t s) {
    if (count <= 0) return;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    switch (nr) {
        case 2: wide_launch<2>(a, outs, count, s, sms); break;
        case 4: wide_launch<4>(a, outs, count, s, sms); break;
        case 6: wide_launch<6>(a, outs, count, s, sms); break;
        case 8: wide_launch<8>(a, outs, count, s, sms); break;
        case 10: wide_launch<10>(a, outs, count, s, sms); break;
        case 12: wide_launch<12>(a, outs, count, s, sms); break;
        case 14: wide_launch<14>(a, outs, count, s, sms); break;
        case 16: wide_launch<16>(a, outs, count, s, sms); break;
        case 18: wide_launch<18>(a, outs, count, s, sms); break;
        case 20: wide_launch<20>(a, outs, count, s, sms); break;
        case 22: wide_launch<22>(a, outs, count, s, sms); break;
        case 24: wide_launch<24>(a, outs, count, s, sms); break;
        case 28: wide_launch<28>(a, outs, count, s, sms); break;
        default: wide_launch<32>(a, outs, count, s, sms); break;
    }
}

namespace {
constexpr int TINY_WARPS = 4;       // warps (independent output streams) per CTA
constexpr int TINY_STAGE = 9216;    // bytes of one chunk buffer; two per warp

__device__ __forceinline__ void cp_async(void *dst, const double2 *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async(void *dst, const float2 *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

__device__ __forceinline__ int pow2_at_least(int n) {
    int p = 1;
    while (p < n) p <<= 1;
    return p;
}

// Descriptors of one output of a warp's sequence: uniform fields, plus the first 32 segments'
// block offsets, widths and vector rows spread over the lanes (lane l: segment e0 + l).
struct TinyOut {
    int o = -1, R = 0, e0 = 0, e1 = 0;
    int64_t moff = 0, voff = 0;
    int w = 0;
};

// STAGE_GATHER for many small outputs (at most 8 NRT rows, bc <= 8 NTL right-hand sides): one
// warp per output, a warp streaming the outputs o = nodes[i] of every TINY_WARPS * gridDim.x-th i.
// The warp's column stream (output by output, segment by segment) is cut into chunks of at most
// wcap columns of one output; every lane issues asynchronous copies (cp.async) of its share of a
// chunk's block columns and vector rows into one of two buffers, so that the next chunk is in
// flight while the current one goes through the FP64 tensor-core MMA (the product kernel's
// consume). The descriptors of the next two outputs are loaded ahead into registers, so that
// issuing a chunk waits on no global load. Outputs are written from the accumulators when their
// last chunk is done (no atomics, fixed order).
template <typename S, int NRT, int NTL, typename VT>
__global__ void __launch_bounds__(TINY_WARPS * 32) k_gather_tiny(RowArgs<S> a, const int32_t *nodes, int count) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, tq = lane & 3;
    unsigned char *const wbuf = smem + 2 * warp * TINY_STAGE;  // this warp's two chunk buffers
    const int bc = a.bc, ldv = conflict_free(bc), bcp = pow2_at_least(bc);
    int bs = 0;
    while (bcp >> (bs + 1)) ++bs;  // log2 of bcp
    const int stride = gridDim.x * TINY_WARPS;
    const double sgn = a.conj ? -1.0 : 1.0;
    const bool scatter = a.y != nullptr;
    constexpr int elem = int(sizeof(S)), vel = int(sizeof(VT));
    // the output sequence of this warp: positions first + j * stride
    const int first = blockIdx.x * TINY_WARPS + warp;
    auto head = [&](int j, TinyOut &d) {  // uniform fields of output j
        const int oi = first + j * stride;
        d.o = -1;
        if (oi < count) {
            d.o = nodes[oi];
            d.R = a.g_rows[d.o];
            d.e0 = a.g_segptr[d.o];
            d.e1 = a.g_segptr[d.o + 1];
        }
    };
    auto segs = [&](TinyOut &d) {  // lane-spread segment fields of output d
        if (d.o >= 0 && lane < d.e1 - d.e0) {
            d.moff = a.g_moff[d.e0 + lane];
            d.w = a.g_w[d.e0 + lane];
            d.voff = a.g_voff[d.e0 + lane];
        }
    };
    // layout of a chunk of an R-row output: block columns (leading dimension ldm) from offset 0,
    // vector rows (stride ldv) from voff; wcap columns, a multiple of 4 when more than 4 fit
    auto layout = [&](int rows, int &ldm, int &wcap, int &voff) {
        ldm = conflict_free(rows);
        wcap = TINY_STAGE / (ldm * elem + ldv * vel);
        if (wcap > 4) wcap &= ~3;
        voff = (wcap * ldm * elem + 15) & ~15;
        while (wcap > 1 && voff + wcap * ldv * vel > TINY_STAGE) {  // the 16-byte rounding of voff
            --wcap;
            voff = (wcap * ldm * elem + 15) & ~15;
        }
    };
    // issuing side: output j (cur, with its segments), j + 1 (nxt, segments in flight) and j + 2
    // (far, uniform fields in flight); position e (absolute segment), column c0 in the segment
    int j = 0;
    TinyOut cur, nxt, far;
    head(0, cur);
    segs(cur);
    head(1, nxt);
    segs(nxt);
    head(2, far);
    int e = cur.e0, c0 = 0;
    // issues the next chunk into b; returns its output (-1: none left), rows, width, last flag
    auto issue = [&](unsigned char *b, int &co, int &cR, int &cW, bool &clast) {
        co = cur.o;
        cR = cur.R;
        cW = 0;
        clast = false;
        if (cur.o < 0) return;
        const int R = cur.R;
        int ldm, wcap, voff;
        layout(R, ldm, wcap, voff);
        S *Ms = reinterpret_cast<S *>(b);
        VT *Vs = reinterpret_cast<VT *>(b + voff);
        const int rp = pow2_at_least(R);
        int rs = 0;
        while (rp >> (rs + 1)) ++rs;  // log2 of rp
        while (e < cur.e1 && cW < wcap) {
            const int l = e - cur.e0;
            int64_t mo, vo;
            int wseg;
            if (l < 32) {
                mo = __shfl_sync(0xffffffffu, cur.moff, l);
                vo = __shfl_sync(0xffffffffu, cur.voff, l);
                wseg = __shfl_sync(0xffffffffu, cur.w, l);
            } else {
                mo = a.g_moff[e];
                vo = a.g_voff[e];
                wseg = a.g_w[e];
            }
            const S *M = mo >= 0 ? a.M + mo : a.M2 + (-1 - mo);
            const int w = wseg - c0 < wcap - cW ? wseg - c0 : wcap - cW;
            const S *msrc = M + int64_t(c0) * R;
            for (int k = lane; k < (w << rs); k += 32) {
                const int r = k & (rp - 1), cc = k >> rs;
                if (r < R) cp_async(Ms + (cW + cc) * ldm + r, msrc + int64_t(cc) * R + r);
            }
            const VT *vsrc = vec_src<VT>(a) + (vo + c0) * a.vs + a.q0;
            for (int k = lane; k < (w << bs); k += 32) {
                const int q = k & (bcp - 1), rr = k >> bs;
                if (q < bc) cp_async(Vs + (cW + rr) * ldv + q, vsrc + int64_t(rr) * a.vs + q);
            }
            cW += w;
            c0 += w;
            if (c0 >= wseg) {
                ++e;
                c0 = 0;
            }
        }
        if (e >= cur.e1) {
            clast = true;
            ++j;
            cur = nxt;
            nxt = far;
            segs(nxt);
            head(j + 2, far);
            e = cur.e0;
            c0 = 0;
        }
    };
    Acc<NRT, NTL> acc;
    acc.zero();
    int co, cR, cW;
    bool clast;
    issue(wbuf, co, cR, cW, clast);
    cp_async_commit();
    for (int k = 0; co >= 0; ++k) {
        int no, nR, nW;
        bool nlast;
        issue(wbuf + ((k + 1) & 1) * TINY_STAGE, no, nR, nW, nlast);
        cp_async_commit();
        cp_async_wait<1>();  // this lane's copies of chunk k have landed
        __syncwarp();        // and every lane's
        TileMap tm;
        tm.init_single(cR);
        int ldm, wcap, voff;
        layout(cR, ldm, wcap, voff);
        consume<S, NRT, NTL, VT>(acc, tm, wbuf + (k & 1) * TINY_STAGE, cW, voff, cR, ldm, bc, ldv, g, tq, sgn);
        if (clast) {
            const int64_t gout = a.g_out[co];
#pragma unroll
            for (int jj = 0; jj < NRT; ++jj) {
                if (jj >= tm.nrt) break;
                const int i = tm.row(jj, g);
                if (i >= cR) continue;
#pragma unroll
                for (int t = 0; t < NTL; ++t)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int qq = t * 8 + 2 * tq + h;
                        if (qq >= bc) continue;
                        double2 v = acc.value(jj * NTL + t, h, sgn);
                        const int col = a.q0 + qq;
                        if (scatter) {
                            double2 *yp = a.y + a.perm[gout + i] + int64_t(col) * a.ldy;
                            double2 out = make_double2(a.alpha.x * v.x - a.alpha.y * v.y,
                                                       a.alpha.x * v.y + a.alpha.y * v.x);
                            if (a.usebeta) {
                                const double2 yo = *yp;
                                out.x += a.beta.x * yo.x - a.beta.y * yo.y;
                                out.y += a.beta.x * yo.y + a.beta.y * yo.x;
                            }
                            *yp = out;
                        } else {
                            VT *d = vec_dst<VT>(a) + (gout + i) * a.vs + col;
                            if (a.accumulate) {
                                const double2 old = widen(*d);
                                v = make_double2(old.x + v.x, old.y + v.y);
                            }
                            *d = narrow<VT>(v);
                        }
                    }
            }
            acc.zero();
        }
        __syncwarp();  // buffer k & 1 is free for chunk k + 2
        co = no;
        cR = nR;
        cW = nW;
        clast = nlast;
    }
    cp_async_wait<0>();
}
}  // namespace

// a single right-hand side keeps the lane-per-row FMA kernel: the tensor-core tiles would be
// 7/8 idle and its single column per memory round trip is then no handicap
bool gather_tiny_fits(int maxrows, int bc) { return maxrows <= 32 && bc >= 2 && bc <= 16; }

template <typename S, typename VT>
void launch_gather_tiny(const RowArgs<S> &a, const int32_t *nodes, int count, cudaStream_t s) {
    if (count <= 0) return;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t sm = size_t(2 * TINY_WARPS) * TINY_STAGE;
    const int need = (count + TINY_WARPS - 1) / TINY_WARPS;
    const int grid = need < 3 * sms ? need : 3 * sms;  // one resident wave of persistent warps
    const int nrt = (a.maxrows + 7) / 8;
    auto go = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
        kern<<<grid, TINY_WARPS * 32, sm, s>>>(a, nodes, count);
    };
    if (a.bc > 8) {
        if (nrt <= 1) go(k_gather_tiny<S, 1, 2, VT>);
        else if (nrt <= 2) go(k_gather_tiny<S, 2, 2, VT>);
        else go(k_gather_tiny<S, 4, 2, VT>);
    } else {
        if (nrt <= 1) go(k_gather_tiny<S, 1, 1, VT>);
        else if (nrt <= 2) go(k_gather_tiny<S, 2, 1, VT>);
        else go(k_gather_tiny<S, 4, 1, VT>);
    }
}

template void launch_gather_tiny<double2, double2>(const RowArgs<double2> &, const int32_t *, int, cudaStream_t);
template void launch_gather_tiny<float2, double2>(const RowArgs<float2> &, const int32_t *, int, cudaStream_t);
template void launch_gather_tiny<float2, float2>(const RowArgs<float2> &, const int32_t *, int, cudaStream_t);

// STAGE_GATHER through the streaming kernel with vectors of type VT
template <typename S, typename VT>
void launch_gather_rows(const RowArgs<S> &a, const int32_t *nodes, int count, cudaStream_t s) {
    if (count <= 0) return;
    const size_t sm = rows_smem_bytes();
    const int MT = (a.maxrows + 7) / 8;
    const int nrt = (MT + NCONS - 1) / NCONS;
    auto go = [&](auto kern) { launch_one<S>(kern, a, nodes, count, s, sm, 0); };
    if (a.bc > 8) {
        if (nrt <= 1) go(k_rows_gather<S, 1, 2, VT>);
        else if (nrt <= 2) go(k_rows_gather<S, 2, 2, VT>);
        else go(k_rows_gather<S, 4, 2, VT>);
    } else {
        if (nrt <= 1) go(k_rows_gather<S, 1, 1, VT>);
        else if (nrt <= 2) go(k_rows_gather<S, 2, 1, VT>);
        else if (nrt <= 4) go(k_rows_gather<S, 4, 1, VT>);
        else go(k_rows_gather<S, 8, 1, VT>);
    }
}

template void launch_gather_rows<double2, double2>(const RowArgs<double2> &, const int32_t *, int, cudaStream_t);
template void launch_gather_rows<float2, double2>(const RowArgs<float2> &, const int32_t *, int, cudaStream_t);
template void launch_gather_rows<float2, float2>(const RowArgs<float2> &, const int32_t *, int, cudaStream_t);

namespace {
template <typename S>
// One warp per block (the blocks are small: a CTA per block left most of its threads idle and
// had one block's index loads in flight at a time)
__global__ void k_copy_blocks(const S *src, const int64_t *soff, const int32_t *sld, const int32_t *rows,
                              const int32_t *cols, const int64_t *doff, int64_t nblocks, S *dst) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = int64_t(gridDim.x) * (blockDim.x >> 5);
    for (int64_t blk = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); blk < nblocks; blk += nw) {
        const int R = rows[blk], Cc = cols[blk], ld = sld[blk];
        const S *in = src + soff[blk];
        S *out = dst + doff[blk];
        for (int e = lane; e < R * Cc; e += 32) {
            const int i = e % R, j = e / R;
            out[e] = in[i + int64_t(j) * ld];
        }
    }
}
}  // namespace

template <typename S>
void launch_copy_blocks(const S *src, const int64_t *soff, const int32_t *sld, const int32_t *rows,
                        const int32_t *cols, const int64_t *doff, int64_t nblocks, S *dst, cudaStream_t s) {
    if (nblocks <= 0) return;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t need = (nblocks + 7) / 8;  // eight warps (blocks) per CTA
    const int grid = int(need < int64_t(sms) * 16 ? need : int64_t(sms) * 16);
    k_copy_blocks<S><<<grid, 256, 0, s>>>(src, soff, sld, rows, cols, doff, nblocks, dst);
}

template void launch_copy_blocks<double2>(const double2 *, const int64_t *, const int32_t *, const int32_t *,
                                          const int32_t *, const int64_t *, int64_t, double2 *, cudaStream_t);

namespace {
template <typename S>
// One warp per block, as k_copy_blocks
__global__ void k_transpose_blocks(const S *in, const int64_t *inoff, const int32_t *rows, const int32_t *cols,
                                   const int64_t *outoff, int64_t nblocks, S *out) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = int64_t(gridDim.x) * (blockDim.x >> 5);
    for (int64_t blk = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); blk < nblocks; blk += nw) {
        const int R = rows[blk], Cc = cols[blk];
        const S *src = in + inoff[blk];
        S *dst = out + outoff[blk];
        for (int e = lane; e < R * Cc; e += 32) {
            const int i = e % R, j = e / R;
            dst[j + int64_t(i) * Cc] = src[e];
        }
    }
}
}  // namespace

template <typename S>
void launch_transpose_blocks(const S *in, const int64_t *inoff, const int32_t *rows, const int32_t *cols,
                             const int64_t *outoff, int64_t nblocks, S *out, cudaStream_t s) {
    if (nblocks <= 0) return;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t need = (nblocks + 7) / 8;  // eight warps (blocks) per CTA
    const int grid = int(need < int64_t(sms) * 16 ? need : int64_t(sms) * 16);
    k_transpose_blocks<S><<<grid, 256, 0, s>>>(in, inoff, rows, cols, outoff, nblocks, out);
}
template void launch_transpose_blocks<double2>(const double2 *, const int64_t *, const int32_t *, const int32_t *,
                                               const int64_t *, int64_t, double2 *, cudaStream_t);
template void launch_transpose_blocks<float2>(const float2 *, const int64_t *, const int32_t *, const int32_t *,
                                              const int64_t *, int64_t, float2 *, cudaStream_t);

}  // namespace nca
