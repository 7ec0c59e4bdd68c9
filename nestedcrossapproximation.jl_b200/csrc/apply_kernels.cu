// Device kernels of the H^2 matrix-vector product (src/nca/aggregate.jl, couple.jl,
// disaggregate.jl and the near-field product of src/nca/petrovgalerkinnca.jl:431-589),
// for a block of b right-hand sides.
//
// Storage per side: one interpolation operator X_p (nrows x rank, column-major) per node;
// the leaf basis is X (test) or X^T (trial), and the transfer matrices of p's children are
// the row slices of X_p in child order. Siblings have consecutive node ids, so the children's
// coefficients form one contiguous slice and every transfer step is a single small GEMM:
//   upward   xhat_p = op(X_p)^T [xhat_c1; xhat_c2; ...]   (leaf: the gathered x slice)
//   coupling yhat_t = sum_s S_ts xhat_s        (reverse: yhat_s = sum_t op(S_ts)^T xhat_t)
//   downward [yhat_c1; ...] += op(X_p) yhat_p
//   leaves   y_t = op(X_t) yhat_t + sum_s op(N_ts) x_s, written straight to the user layout.
// Every stage is a gather (the reverse coupling and the transposed near field read the
// trial-side CSR transposes), so no atomics are used and results are bitwise reproducible.
// Vectors are laid out point-major with the right-hand sides contiguous: v[i * b + q].
#include <cuda_runtime.h>

#include <cstdint>

#include "apply_kernels.cuh"

namespace nca {

namespace {

constexpr int NT = 256;

__device__ __forceinline__ double2 ld_c(const double2 *p) { return *p; }
__device__ __forceinline__ double2 ld_c(const float2 *p) {
    float2 v = *p;
    return make_double2(v.x, v.y);
}

template <typename C>
struct Cx;
template <>
struct Cx<double2> {
    __device__ static double2 zero() { return make_double2(0.0, 0.0); }
    __device__ static double2 from(double2 v) { return v; }
    __device__ static double2 fma(double2 a, double2 b, double2 c) {
        return make_double2(::fma(a.x, b.x, ::fma(-a.y, b.y, c.x)), ::fma(a.x, b.y, ::fma(a.y, b.x, c.y)));
    }
};
template <>
struct Cx<float2> {
    __device__ static float2 zero() { return make_float2(0.f, 0.f); }
    __device__ static float2 from(double2 v) { return make_float2(float(v.x), float(v.y)); }
    __device__ static float2 fma(float2 a, float2 b, float2 c) {
        return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
    }
};

__device__ __forceinline__ double2 to_d(double2 v) { return v; }
__device__ __forceinline__ double2 to_d(float2 v) { return make_double2(v.x, v.y); }

template <typename C>
__device__ __forceinline__ C conj_if(C a, bool c) {
    if (c) a.y = -a.y;
    return a;
}

// Shared-memory plan of one block product: output accumulator M x bc (double2), a tile of the
// matrix (element type C) and a tile of the right operand (C).
struct Smem {
    double2 *acc;
    unsigned char *a;
    unsigned char *b;
    int kc;  // columns of the inner dimension per tile
};

// acc(row, q) += sum_k opA(row, k) * B(k, q), rows < M, inner < K, q < bc.
// A (element S, global memory): TRANS ? A[k + row * lda] : A[row + k * lda]; conj if conjA.
// B (global, double2): B[k * bstride + q].
template <typename S, typename C, bool TRANS>
__device__ void block_gemm(const S *A, int64_t lda, int M, int K, bool conjA, const double2 *B,
                           int bstride, int bc, const Smem &sm) {
    C *As = reinterpret_cast<C *>(sm.a);
    C *Bs = reinterpret_cast<C *>(sm.b);
    const int tid = threadIdx.x;
    for (int k0 = 0; k0 < K; k0 += sm.kc) {
        const int kc = min(sm.kc, K - k0);
        // tile of A as M x kc column-major in smem (opA(row, k0 + kk) at As[row + kk * M])
        if (!TRANS) {
            for (int e = tid; e < M * kc; e += NT) {
                int row = e % M, kk = e / M;
                As[e] = conj_if(Cx<C>::from(ld_c(A + row + (k0 + kk) * lda)), conjA);
            }
        } else {
            for (int e = tid; e < M * kc; e += NT) {
                int kk = e % kc, row = e / kc;
                As[row + kk * M] = conj_if(Cx<C>::from(ld_c(A + (k0 + kk) + row * lda)), conjA);
            }
        }
        for (int e = tid; e < kc * bc; e += NT) {
            int kk = e / bc, q = e % bc;
            Bs[e] = Cx<C>::from(B[int64_t(k0 + kk) * bstride + q]);
        }
        __syncthreads();
        for (int e = tid; e < M * bc; e += NT) {
            int row = e / bc, q = e % bc;
            C s = Cx<C>::zero();
            for (int kk = 0; kk < kc; ++kk) s = Cx<C>::fma(As[row + kk * M], Bs[kk * bc + q], s);
            double2 d = to_d(s);
            sm.acc[e].x += d.x;
            sm.acc[e].y += d.y;
        }
        __syncthreads();
    }
}

__device__ Smem carve(unsigned char *base, int mcap, int bc, int tile_bytes, int elem) {
    Smem s;
    s.acc = reinterpret_cast<double2 *>(base);
    size_t off = sizeof(double2) * size_t(mcap) * bc;
    s.a = base + off;
    s.b = s.a + tile_bytes;
    s.kc = tile_bytes / (elem * (mcap > bc ? mcap : bc));
    if (s.kc < 1) s.kc = 1;
    return s;
}

__device__ void zero_acc(double2 *acc, int n) {
    for (int e = threadIdx.x; e < n; e += NT) acc[e] = make_double2(0.0, 0.0);
    __syncthreads();
}

}  // namespace

size_t apply_smem_bytes(int mcap, int bc, int tile_bytes) {
    return sizeof(double2) * size_t(mcap) * bc + 2 * size_t(tile_bytes);
}

__global__ void k_gather(const double2 *x, int64_t ldx, const int32_t *perm, int64_t n, int b,
                         double2 *xt) {
    int64_t total = n * b;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
         e += int64_t(gridDim.x) * blockDim.x) {
        int64_t i = e / b;
        int q = int(e % b);
        xt[e] = x[perm[i] + q * ldx];
    }
}

template <typename S, typename C>
__global__ void __launch_bounds__(NT) k_up(SweepArgs<S> a, const int32_t *nodes, int mcap,
                                           int tile_bytes) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int p = nodes[blockIdx.x];
    const int m = a.nrows[p], r = a.rank[p];
    const double2 *src = a.nchildren[p] == 0 ? a.xt + int64_t(a.begin[p]) * a.b
                                             : a.coef + a.cptr[a.firstchild[p]] * a.b;
    double2 *dst = a.coef + a.cptr[p] * a.b;
    const S *X = a.X + a.xoff[p];
    for (int q0 = 0; q0 < a.b; q0 += 16) {
        const int bc = min(16, a.b - q0);
        Smem sm = carve(smem, mcap, bc, tile_bytes, sizeof(C));
        zero_acc(sm.acc, r * bc);
        block_gemm<S, C, true>(X, m, r, m, a.conj, src + q0, a.b, bc, sm);
        for (int e = threadIdx.x; e < r * bc; e += NT) dst[int64_t(e / bc) * a.b + q0 + e % bc] = sm.acc[e];
        __syncthreads();
    }
}

template <typename S, typename C>
__global__ void __launch_bounds__(NT) k_down(SweepArgs<S> a, const int32_t *nodes, int mcap,
                                             int tile_bytes) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int p = nodes[blockIdx.x];
    const int m = a.nrows[p], r = a.rank[p];
    const double2 *src = a.coef + a.cptr[p] * a.b;
    double2 *dst = a.coef + a.cptr[a.firstchild[p]] * a.b;
    const S *X = a.X + a.xoff[p];
    for (int q0 = 0; q0 < a.b; q0 += 16) {
        const int bc = min(16, a.b - q0);
        Smem sm = carve(smem, mcap, bc, tile_bytes, sizeof(C));
        for (int e = threadIdx.x; e < m * bc; e += NT) sm.acc[e] = dst[int64_t(e / bc) * a.b + q0 + e % bc];
        __syncthreads();
        block_gemm<S, C, false>(X, m, m, r, a.conj, src + q0, a.b, bc, sm);
        for (int e = threadIdx.x; e < m * bc; e += NT) dst[int64_t(e / bc) * a.b + q0 + e % bc] = sm.acc[e];
        __syncthreads();
    }
}

template <typename S, typename C>
__global__ void __launch_bounds__(NT) k_couple(CoupleArgs<S> a, const int32_t *nodes, int mcap,
                                               int tile_bytes) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int o = nodes[blockIdx.x];  // output node (test node forward, trial node reverse)
    const int ko = a.rank_out[o];
    double2 *dst = a.yhat + a.cptr_out[o] * a.b;
    for (int q0 = 0; q0 < a.b; q0 += 16) {
        const int bc = min(16, a.b - q0);
        Smem sm = carve(smem, mcap, bc, tile_bytes, sizeof(C));
        zero_acc(sm.acc, ko * bc);
        for (int k = a.ptr[o]; k < a.ptr[o + 1]; ++k) {
            const int pair = a.pairs ? a.pairs[k] : k;
            const int other = a.other[k];
            const int ki = a.rank_in[other];
            if (ki == 0) continue;
            const S *Cm = a.C + a.coff[pair];
            const double2 *src = a.xhat + a.cptr_in[other] * a.b + q0;
            if (!a.reverse)
                block_gemm<S, C, false>(Cm, ko, ko, ki, false, src, a.b, bc, sm);
            else
                block_gemm<S, C, true>(Cm, ki, ko, ki, a.conj, src, a.b, bc, sm);
        }
        for (int e = threadIdx.x; e < ko * bc; e += NT) dst[int64_t(e / bc) * a.b + q0 + e % bc] = sm.acc[e];
        __syncthreads();
    }
}

template <typename S, typename C>
__global__ void __launch_bounds__(NT) k_leaves(LeafArgs<S> a, const int32_t *leaves, int mcap,
                                               int tile_bytes) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int t = leaves[blockIdx.x];
    const int mt = a.end[t] - a.begin[t];
    const int r = a.rank[t];
    for (int q0 = 0; q0 < a.b; q0 += 16) {
        const int bc = min(16, a.b - q0);
        Smem sm = carve(smem, mcap, bc, tile_bytes, sizeof(C));
        zero_acc(sm.acc, mt * bc);
        if (r > 0 && a.nrows[t] == mt)
            block_gemm<S, C, false>(a.X + a.xoff[t], mt, mt, r, a.conj, a.yhat + a.cptr[t] * a.b + q0,
                                    a.b, bc, sm);
        for (int k = a.nptr[t]; k < a.nptr[t + 1]; ++k) {
            const int o = a.nnodes[k];
            const int mo = a.o_end[o] - a.o_begin[o];
            const double2 *src = a.xt + int64_t(a.o_begin[o]) * a.b + q0;
            if (!a.reverse) {
                // forward: N_ts is mt x ms at column offset coloff of t's row block
                const S *Nm = a.N + a.noff[t] + int64_t(a.coloff[k]) * mt;
                block_gemm<S, C, false>(Nm, mt, mt, mo, false, src, a.b, bc, sm);
            } else {
                // transposed: N_{o,t} is mo x mt at column offset coloff of o's row block
                const S *Nm = a.N + a.noff[o] + int64_t(a.coloff[k]) * mo;
                block_gemm<S, C, true>(Nm, mo, mt, mo, a.conj, src, a.b, bc, sm);
            }
        }
        const double2 al = a.alpha, be = a.beta;
        const bool usebeta = be.x != 0.0 || be.y != 0.0;
        for (int e = threadIdx.x; e < mt * bc; e += NT) {
            const int i = e / bc, q = q0 + e % bc;
            double2 v = sm.acc[e];
            double2 out = make_double2(al.x * v.x - al.y * v.y, al.x * v.y + al.y * v.x);
            double2 *yp = a.y + a.perm[a.begin[t] + i] + int64_t(q) * a.ldy;
            if (usebeta) {
                double2 yo = *yp;
                out.x += be.x * yo.x - be.y * yo.y;
                out.y += be.x * yo.y + be.y * yo.x;
            }
            *yp = out;
        }
        __syncthreads();
    }
}

namespace {
// The attribute is per device and per kernel; setting it costs far less than a launch.
template <typename K>
void raise_smem(K kernel, size_t bytes) {
    if (bytes > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
}
}  // namespace

template <typename S>
void launch_up(const SweepArgs<S> &a, const int32_t *nodes, int count, int mcap, int tile, cudaStream_t s) {
    size_t sm = apply_smem_bytes(mcap, a.b < 16 ? a.b : 16, tile);
    raise_smem(k_up<S, S>, sm);
    k_up<S, S><<<count, NT, sm, s>>>(a, nodes, mcap, tile);
}
template <typename S>
void launch_down(const SweepArgs<S> &a, const int32_t *nodes, int count, int mcap, int tile, cudaStream_t s) {
    size_t sm = apply_smem_bytes(mcap, a.b < 16 ? a.b : 16, tile);
    raise_smem(k_down<S, S>, sm);
    k_down<S, S><<<count, NT, sm, s>>>(a, nodes, mcap, tile);
}
template <typename S>
void launch_couple(const CoupleArgs<S> &a, const int32_t *nodes, int count, int mcap, int tile, cudaStream_t s) {
    size_t sm = apply_smem_bytes(mcap, a.b < 16 ? a.b : 16, tile);
    raise_smem(k_couple<S, S>, sm);
    k_couple<S, S><<<count, NT, sm, s>>>(a, nodes, mcap, tile);
}
template <typename S>
void launch_leaves(const LeafArgs<S> &a, const int32_t *nodes, int count, int mcap, int tile, cudaStream_t s) {
    size_t sm = apply_smem_bytes(mcap, a.b < 16 ? a.b : 16, tile);
    raise_smem(k_leaves<S, S>, sm);
    k_leaves<S, S><<<count, NT, sm, s>>>(a, nodes, mcap, tile);
}

template void launch_up<double2>(const SweepArgs<double2> &, const int32_t *, int, int, int, cudaStream_t);
template void launch_up<float2>(const SweepArgs<float2> &, const int32_t *, int, int, int, cudaStream_t);
template void launch_down<double2>(const SweepArgs<double2> &, const int32_t *, int, int, int, cudaStream_t);
template void launch_down<float2>(const SweepArgs<float2> &, const int32_t *, int, int, int, cudaStream_t);
template void launch_couple<double2>(const CoupleArgs<double2> &, const int32_t *, int, int, int, cudaStream_t);
template void launch_couple<float2>(const CoupleArgs<float2> &, const int32_t *, int, int, int, cudaStream_t);
template void launch_leaves<double2>(const LeafArgs<double2> &, const int32_t *, int, int, int, cudaStream_t);
template void launch_leaves<float2>(const LeafArgs<float2> &, const int32_t *, int, int, int, cudaStream_t);

}  // namespace nca
