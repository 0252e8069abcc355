// Sparse adjacency products for the Frank-Wolfe gradient (cugal/pred.py:54-74,
// cugal/adjacency.py:128-156, cuda_kernels/adjacency.cu:77-150).
//
// The reference builds the gradient of the symmetric case as
// B.mul(A.mul(P).T).T * -2 with two cuSPARSE SpMM calls (a handle, a value
// vector and a buffer allocated per call), then adds the distance and the
// lambda term in two more n^2 passes.  Here:
//
//   kernel 1:  T = A P, each output tile transposed through shared memory on
//              the way out, so Tt = (A P)^T is row-major;
//   kernel 2:  Y = B Tt = (A P B)^T (A, B symmetric), transposed back in
//              shared memory, and the epilogue writes
//              out = s * (-2 APB + ||Fs_i - Ft_j|| + c lambda (1 - 2P)) + U_i + V_j
//              in one pass (distance recomputed from the 4 feature columns, no
//              n^2 distance matrix is ever stored).
//
// Both kernels gather rows of the dense operand with warp-wide 512-byte float4
// loads.  The grid walks output tiles panel-major (blockIdx.x = row tile,
// blockIdx.y = 128-column panel), so the CTAs in flight share one panel of the
// dense operand (n x 128 x 4 bytes, 16 MB at n = 32768) and the gathers hit L2.
// The 32 x 128 output tile sits in shared memory as 16-byte chunks whose chunk
// index is XOR-swizzled by (row mod 8): a warp stores a gathered row as one
// 16-byte store per lane, and reads four columns of 32 rows (the transposed
// orientation) as one 16-byte load per lane, both without bank conflicts.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdint>
#include <type_traits>

#include "fugal_common.cuh"
#include "fugal_host.h"

namespace fugal {

constexpr int kTileRows = 32;     // gathered output rows per CTA
constexpr int kTileCols = 128;    // columns per CTA (32 lanes x float4)
constexpr int kSpmmThreads = 256; // 8 warps, 4 rows each
constexpr int kChunks = kTileCols / 4;  // 16-byte chunks per tile row

// The tile: kTileRows rows of kChunks float4 chunks; chunk q of row r is stored
// at position q ^ (r & 7).
struct Tile {
    float4 c[kTileRows][kChunks];
    __device__ __forceinline__ float4& at(int r, int q) { return c[r][q ^ (r & 7)]; }
};

// 4 consecutive floats of row k starting at column c: one 16-byte load when the
// rows are 16-byte aligned (VEC), else scalar loads guarded by n.  (Loads that
// skip L1 allocation, ld.global.nc.L1::no_allocate, made the pair of gradient
// kernels 50% slower at n = 32768.)
// Row offset k * ldx as one 32 x 32 -> 64-bit multiply (k >= 0 and ldx < 2^32).
__device__ __forceinline__ unsigned long long row_offset(int k, long long ldx) {
    return static_cast<unsigned long long>(static_cast<unsigned>(k)) * static_cast<unsigned>(ldx);
}

template <bool VEC>
__device__ __forceinline__ float4 load4(const float* __restrict__ X, long long ldx, int k, int c, int n) {
    const float* p = X + row_offset(k, ldx) + c;
    if (VEC) return __ldg(reinterpret_cast<const float4*>(p));
    float4 v;
    v.x = __ldg(p);
    v.y = c + 1 < n ? __ldg(p + 1) : 0.f;
    v.z = c + 2 < n ? __ldg(p + 2) : 0.f;
    v.w = c + 3 < n ? __ldg(p + 3) : 0.f;
    return v;
}

// acc = sum over k in N(row) of X[k][c .. c+3] (4 columns per lane), U gathers in
// flight per lane.
template <bool VEC, int U>
__device__ __forceinline__ float4 gather_row(const int* __restrict__ rp, const int* __restrict__ col,
                                             const float* __restrict__ X, long long ldx, int n, int row, int c,
                                             bool c_ok) {
    // two packed FP32x2 accumulators (fadd.f32x2); each column still sums its
    // neighbours one by one in CSR order
    float2 lo = make_float2(0.f, 0.f), hi = make_float2(0.f, 0.f);
    auto add = [&](const float4& v) {
        lo = __fadd2_rn(lo, make_float2(v.x, v.y));
        hi = __fadd2_rn(hi, make_float2(v.z, v.w));
    };
    const int lane = threadIdx.x & 31;
    const float* Xc = X + c;  // this lane's columns; rows are offset from here
    const int rs = rp[row], re = rp[row + 1];
    for (int e = rs; e < re; e += 32) {
        const int cnt = min(32, re - e);
        const int idx = (lane < cnt) ? col[e + lane] : 0;
        int q = 0;
        for (; q + U <= cnt; q += U) {
            int k[U];
#pragma unroll
            for (int t = 0; t < U; ++t) k[t] = __shfl_sync(0xffffffffu, idx, q + t);
            if (c_ok) {
                float4 v[U];
#pragma unroll
                for (int t = 0; t < U; ++t) v[t] = load4<VEC>(Xc, ldx, k[t], 0, n - c);
#pragma unroll
                for (int t = 0; t < U; ++t) add(v[t]);
            }
        }
        for (; q < cnt; ++q) {
            const int k = __shfl_sync(0xffffffffu, idx, q);
            if (c_ok) add(load4<VEC>(Xc, ldx, k, 0, n - c));
        }
    }
    return make_float4(lo.x, lo.y, hi.x, hi.y);
}

// Fill the tile with the gathered rows r0 .. r0+31 of A X for columns c0 .. c0+127
// (lane l: chunk l of each row).
template <bool VEC, int U>
__device__ __forceinline__ void gather_tile(const int* __restrict__ rp, const int* __restrict__ col,
                                            const float* __restrict__ X, long long ldx, int n, int r0, int c0,
                                            Tile& tile, float sign) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int c = c0 + lane * 4;
    const bool c_ok = c < n;
    for (int rr = warp; rr < kTileRows; rr += kSpmmThreads / 32) {
        const int row = r0 + rr;
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        if (row < n) acc = gather_row<VEC, U>(rp, col, X, ldx, n, row, c, c_ok);
        tile.at(rr, lane) = make_float4(sign * acc.x, sign * acc.y, sign * acc.z, sign * acc.w);
    }
}

// Tt[c][r] = (A X)[r][c]  (transposed store), or out[r][c] = sign (A X)[r][c] (direct store).
template <bool VEC, int U = 4>
__global__ void __launch_bounds__(kSpmmThreads) spmm_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                                            const float* __restrict__ X, long long ldx, int n,
                                                            float* __restrict__ out, long long ldo, int transpose,
                                                            float sign) {
    __shared__ Tile tile;
    const int r0 = blockIdx.x * kTileRows;
    const int c0 = blockIdx.y * kTileCols;
    gather_tile<VEC, U>(rp, col, X, ldx, n, r0, c0, tile, sign);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (transpose) {
        // rows c0+4q .. c0+4q+3 of out get the 32 values of columns 4q .. 4q+3 of the
        // tile: lane l reads chunk q of tile row l
        const int rg = r0 + lane;
        for (int q = warp; q < kChunks; q += kSpmmThreads / 32) {
            const float4 v = tile.at(lane, q);
            const int cg = c0 + 4 * q;
            if (rg < n) {
                float* o = out + row_offset(cg, ldo) + rg;
                if (cg + 0 < n) o[0] = v.x;
                if (cg + 1 < n) o[ldo] = v.y;
                if (cg + 2 < n) o[2 * ldo] = v.z;
                if (cg + 3 < n) o[3 * ldo] = v.w;
            }
        }
    } else {
        for (int rr = warp; rr < kTileRows; rr += kSpmmThreads / 32) {
            const int rg = r0 + rr;
            if (rg >= n) continue;
            const float4 v = tile.at(rr, lane);
            const int cg = c0 + 4 * lane;
            float* o = out + static_cast<size_t>(rg) * ldo + cg;
            if (cg + 3 < n && (reinterpret_cast<uintptr_t>(o) & 15u) == 0) {
                *reinterpret_cast<float4*>(o) = v;
            } else {
                if (cg + 0 < n) o[0] = v.x;
                if (cg + 1 < n) o[1] = v.y;
                if (cg + 2 < n) o[2] = v.z;
                if (cg + 3 < n) o[3] = v.w;
            }
        }
    }
}

struct EpilogueArgs {
    const float* P;
    long long ldp;
    const float* fs;  // n x 4 (nullable)
    const float* ft;
    const float* D;   // stored distances (nullable; used when fs is null)
    long long ldd;
    double lam;       // lambda * lambda_scale
    double out_scale;
    const double* U;  // nullable
    const double* V;
    float* out;
    long long ldo;
    float2* colpart;  // COLSTATS: [n / 128 panels][ldc] base-2 (max, sum) of out's columns
    long long ldc;
};

// Y = B Tt = (APB)^T over the tile (rows j0.., cols i0..), then the gradient
// epilogue in (i, j) orientation: lane l takes j = j0 + l, and warp w the tile
// columns i0 + 4q .. i0 + 4q + 3 for q = w, w + 8, w + 16, w + 24 (one 16-byte
// tile read per q), so every global access is a 128-byte row segment.  The P
// term is skipped when lambda is 0 (its factor).  COLSTATS: the CTA also
// reduces, for each of its 32 output columns j, the 128 values it wrote over
// rows i0 .. i0+127 to a base-2 (max, sum) pair, x = out log2 e: M = max x,
// S = sum 2^(x - M), stored at colpart[blockIdx.y][j] (the first column update
// of the Sinkhorn solve merges them instead of reading the cost again).
// PK: chunks of four in-range columns with features take a packed path -- the
// FP32 arithmetic of two columns per FP32x2 instruction (the same IEEE operations
// in the same order, so the same results) and the row duals read from shared
// memory; other chunks take the scalar path.
// SQ: the distance's square root as sqrt.approx, the form the reference's
// distance kernel is built with (--use_fast_math, cuda_kernels/setup.py:19),
// instead of the IEEE-rounded one.
template <bool COLSTATS, int U = 4, int MINB = 6, bool PK = true, bool SQ = false>
__global__ void __launch_bounds__(kSpmmThreads, MINB) gradient_kernel(const int* __restrict__ rp,
                                                                const int* __restrict__ col,
                                                                const float* __restrict__ Tt, long long ldt, int n,
                                                                const EpilogueArgs ep) {
    constexpr int kWarps = kSpmmThreads / 32;
    __shared__ Tile tile;
    __shared__ float4 fi[kTileCols];
    __shared__ float4 fj[kTileRows];
    __shared__ float2 cst[COLSTATS ? kWarps : 1][kTileRows];
    __shared__ double us[kTileCols];
    const int j0 = blockIdx.x * kTileRows;   // gathered rows: target nodes j
    const int i0 = blockIdx.y * kTileCols;   // lanes: source nodes i
    const bool has_f = ep.fs != nullptr;
    if constexpr (PK) {
        for (int q = threadIdx.x; q < kTileCols; q += kSpmmThreads)
            us[q] = (ep.U != nullptr && i0 + q < n) ? ep.U[i0 + q] : 0.0;
    }
    if (has_f) {
        for (int q = threadIdx.x; q < kTileCols; q += kSpmmThreads)
            fi[q] = (i0 + q < n) ? reinterpret_cast<const float4*>(ep.fs)[i0 + q] : make_float4(0, 0, 0, 0);
        for (int q = threadIdx.x; q < kTileRows; q += kSpmmThreads)
            fj[q] = (j0 + q < n) ? reinterpret_cast<const float4*>(ep.ft)[j0 + q] : make_float4(0, 0, 0, 0);
    }
    gather_tile<true, U>(rp, col, Tt, ldt, n, j0, i0, tile, 1.0f);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int j = j0 + lane;
    if (!COLSTATS && j >= n) return;
    const double vj = (ep.V && j < n) ? ep.V[j] : 0.0;
    const float4 f2 = has_f ? fj[lane] : make_float4(0, 0, 0, 0);
    const float lam = static_cast<float>(ep.lam);
    const bool use_p = lam != 0.f;
    float xmax = -INFINITY;
    for (int q = warp; q < kChunks; q += kWarps) {
        if (i0 + 4 * q >= n || j >= n) break;
        if (PK && has_f && i0 + 4 * q + 3 < n) {
            const float4 apb4 = tile.at(lane, q);
            const float2 m2 = make_float2(-2.0f, -2.0f);
            float2 g2[2] = {__fmul2_rn(m2, make_float2(apb4.x, apb4.y)), __fmul2_rn(m2, make_float2(apb4.z, apb4.w))};
            const int ib = i0 + 4 * q;
            if (use_p) {
                const float* pc = ep.P + row_offset(ib, ep.ldp) + j;
                const float2 lam2 = make_float2(lam, lam), one2 = make_float2(1.0f, 1.0f);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const float2 p2 = make_float2(pc[(2 * h) * ep.ldp], pc[(2 * h + 1) * ep.ldp]);
                    // lam (1 - 2p): 1 + (-2p) is 1 - 2p exactly
                    g2[h] = __fadd2_rn(g2[h], __fmul2_rn(lam2, __fadd2_rn(one2, __fmul2_rn(m2, p2))));
                }
            } else {
#pragma unroll
                for (int h = 0; h < 2; ++h) g2[h] = __fadd2_rn(g2[h], make_float2(0.f, 0.f));
            }
            float o[4];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const float4 fa = fi[4 * q + 2 * h], fb = fi[4 * q + 2 * h + 1];
                const float2 d0 = __fadd2_rn(make_float2(fa.x, fb.x), make_float2(-f2.x, -f2.x));
                const float2 d1 = __fadd2_rn(make_float2(fa.y, fb.y), make_float2(-f2.y, -f2.y));
                const float2 d2 = __fadd2_rn(make_float2(fa.z, fb.z), make_float2(-f2.z, -f2.z));
                const float2 d3 = __fadd2_rn(make_float2(fa.w, fb.w), make_float2(-f2.w, -f2.w));
                float2 ss = __fmul2_rn(d0, d0);
                ss = __ffma2_rn(d1, d1, ss);
                ss = __ffma2_rn(d2, d2, ss);
                ss = __ffma2_rn(d3, d3, ss);
                float2 dist;
                if constexpr (SQ) {
                    asm("sqrt.approx.f32 %0, %1;" : "=f"(dist.x) : "f"(ss.x));
                    asm("sqrt.approx.f32 %0, %1;" : "=f"(dist.y) : "f"(ss.y));
                } else {
                    dist = make_float2(__fsqrt_rn(ss.x), __fsqrt_rn(ss.y));
                }
                const float2 g = __fadd2_rn(g2[h], dist);
                o[2 * h] = static_cast<float>(ep.out_scale * static_cast<double>(g.x) + (us[4 * q + 2 * h] + vj));
                o[2 * h + 1] =
                    static_cast<float>(ep.out_scale * static_cast<double>(g.y) + (us[4 * q + 2 * h + 1] + vj));
            }
            float* oc = ep.out + row_offset(ib, ep.ldo) + j;
#pragma unroll
            for (int t = 0; t < 4; ++t) oc[t * ep.ldo] = o[t];
            if constexpr (COLSTATS) {
                const float4 x = make_float4(o[0] * kLog2e, o[1] * kLog2e, o[2] * kLog2e, o[3] * kLog2e);
                xmax = fmaxf(xmax, fmaxf(fmaxf(x.x, x.y), fmaxf(x.z, x.w)));
                tile.at(lane, q) = x;
            }
            continue;
        }
        const float4 apb4 = tile.at(lane, q);
        const float apbs[4] = {apb4.x, apb4.y, apb4.z, apb4.w};
        float xs[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int ii = 4 * q + t;
            const int i = i0 + ii;
            xs[t] = -INFINITY;
            if (i >= n) continue;
            // The gradient itself in FP32, as the reference computes it (SpMM, distance,
            // regularize: cugal/pred.py:54-74, distance.cu:11-53, regularize.cu:10-39) ...
            float reg = 0.f;
            if (use_p) {
                const float p = ep.P[static_cast<size_t>(i) * ep.ldp + j];
                reg = __fmul_rn(lam, __fsub_rn(1.0f, __fmul_rn(2.0f, p)));
            }
            float g = __fadd_rn(__fmul_rn(-2.0f, apbs[t]), reg);
            if (has_f) {
                const float4 f1 = fi[ii];
                const float d0 = __fsub_rn(f1.x, f2.x), d1 = __fsub_rn(f1.y, f2.y);
                const float d2 = __fsub_rn(f1.z, f2.z), d3 = __fsub_rn(f1.w, f2.w);
                const float ss = __fmaf_rn(d3, d3, __fmaf_rn(d2, d2, __fmaf_rn(d1, d1, __fmul_rn(d0, d0))));
                float dist;
                if constexpr (SQ) asm("sqrt.approx.f32 %0, %1;" : "=f"(dist) : "f"(ss));
                else dist = __fsqrt_rn(ss);
                g = __fadd_rn(g, dist);
            } else if (ep.D != nullptr) {
                g = __fadd_rn(g, ep.D[static_cast<size_t>(i) * ep.ldd + j]);
            }
            // ... and its combination with the accumulated duals in FP64: the terms are
            // O(1/reg) and cancel to O(1), which FP32 would not resolve.
            const double ui = ep.U ? ep.U[i] : 0.0;
            const float o = static_cast<float>(ep.out_scale * static_cast<double>(g) + (ui + vj));
            ep.out[static_cast<size_t>(i) * ep.ldo + j] = o;
            xs[t] = o * kLog2e;
            xmax = fmaxf(xmax, xs[t]);
        }
        if constexpr (COLSTATS) {
            // the chunk this thread just consumed keeps x = out log2 e for the sum below
            tile.at(lane, q) = make_float4(xs[0], xs[1], xs[2], xs[3]);
        }
    }
    if constexpr (COLSTATS) {
        // second pass over the same tile chunks (this thread's own, no barrier needed);
        // chunks past n hold -inf and add 0
        float sum = 0.f;
        if (xmax != -INFINITY) {
            for (int q = warp; q < kChunks && i0 + 4 * q < n; q += kWarps) {
                const float4 x = tile.at(lane, q);
                sum += ex2(x.x - xmax);
                sum += ex2(x.y - xmax);
                sum += ex2(x.z - xmax);
                sum += ex2(x.w - xmax);
            }
        }
        cst[warp][lane] = make_float2(xmax, sum);
        __syncthreads();
        if (warp == 0 && j < n) {
            float M = -INFINITY;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) M = fmaxf(M, cst[w][lane].x);
            float S = 0.f;
            if (M != -INFINITY) {
#pragma unroll
                for (int w = 0; w < kWarps; ++w) {
                    const float2 ps = cst[w][lane];
                    if (ps.x != -INFINITY) S += ps.y * ex2(ps.x - M);
                }
            }
            ep.colpart[static_cast<size_t>(blockIdx.y) * ep.ldc + j] = make_float2(M, S);
        }
    }
}

// Fixed-point refresh of the structural term: the gather of gradient_kernel
// (Y = B Tt = (A P B)^T over the tile), stored as Mq[i][j] = round(APB * scale)
// in int64 (lane = j, so each store is a 256-byte row segment).  APB >= 0; a
// value at or above 2^52 (or not finite) sets flags[1] and stores 0.
template <int U = 4>
__global__ void __launch_bounds__(kSpmmThreads) structural_refresh_kernel(const int* __restrict__ rp,
                                                                          const int* __restrict__ col,
                                                                          const float* __restrict__ Tt, long long ldt,
                                                                          int n, long long* __restrict__ Mq,
                                                                          long long ldm, double scale, int* flags) {
    __shared__ Tile tile;
    const int j0 = blockIdx.x * kTileRows;
    const int i0 = blockIdx.y * kTileCols;
    gather_tile<true, U>(rp, col, Tt, ldt, n, j0, i0, tile, 1.0f);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int j = j0 + lane;
    if (j >= n) return;
    bool bad = false;
    for (int q = warp; q < kChunks; q += kSpmmThreads / 32) {
        const int ib = i0 + 4 * q;
        if (ib >= n) break;
        const float4 a = tile.at(lane, q);
        const float av[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            if (ib + t >= n) break;
            const double x = static_cast<double>(av[t]) * scale;
            long long m = 0;
            if (x < 4503599627370496.0 && x >= 0.0) m = __double2ll_rn(x);
            else bad = true;
            Mq[row_offset(ib + t, ldm) + j] = m;
        }
    }
    if (bad) atomicOr(&flags[1], 1);
}

// (float)(m * scale) for a fixed-point value 0 <= m < 2^52: OR-ing m into the
// mantissa of 2^52 gives the double 2^52 + m exactly, and one fused multiply-add,
// (2^52 + m) scale - 2^52 scale, rounds m * scale once (no 64-bit integer
// convert).
__device__ __forceinline__ float fixed_to_float(long long m, double scale, double bias) {
    const double x = __longlong_as_double(0x4330000000000000ll | m);
    return __double2float_rn(fma(x, scale, bias));
}

// The gradient of gradient_kernel with APB read from the fixed-point structural
// term (apb = (float)(Mq * m_scale)) instead of gathered: an elementwise pass.
// CTA tile: 128 rows (i0 = 128 blockIdx.y, the column-statistics panel) x 32 CPT
// columns (j0 = 32 CPT blockIdx.x); lane l owns the CPT consecutive columns
// j0 + CPT l ..., warp w the rows i0 + w + 8r, so every warp access is one
// contiguous row segment (256 CPT bytes of Mq, 128 CPT of P and of the cost).
// Each thread loads 8 / CPT rows before computing any of them (bytes in flight);
// the tile's features and duals sit in shared memory.  The per-column (max, sum)
// in base 2 is kept online (one ex2 per element) and merged over the warps in
// shared memory.  SHIFT: Mq is also written back divided by 2^shift (rounded
// half up).  SQ: the distance's square root as sqrt.approx, as gradient_kernel's.
constexpr int kStructThreads = 256;
constexpr int kStructRows = 128;
// 2 columns per thread: 4 columns (2 rows in flight, 3 CTAs per SM) measured
// 4.13 against 3.91 ms per FW step at n = 32768
constexpr int kStructCpt = 2;

template <int CPT> struct StructVec;
template <> struct StructVec<2> {
    static __device__ __forceinline__ void load_m(const long long* p, long long (&m)[2]) {
        const longlong2 a = *reinterpret_cast<const longlong2*>(p);
        m[0] = a.x;
        m[1] = a.y;
    }
    static __device__ __forceinline__ void load_p(const float* p, float (&v)[2]) {
        const float2 a = *reinterpret_cast<const float2*>(p);
        v[0] = a.x;
        v[1] = a.y;
    }
    static __device__ __forceinline__ void store_o(float* p, const float (&o)[2]) {
        *reinterpret_cast<float2*>(p) = make_float2(o[0], o[1]);
    }
    static __device__ __forceinline__ void store_m(long long* p, const long long (&m)[2]) {
        *reinterpret_cast<longlong2*>(p) = make_longlong2(m[0], m[1]);
    }
};
template <bool COLSTATS, bool SHIFT, bool SQ, int CPT>
__global__ void __launch_bounds__(kStructThreads, 4) gradient_structural_kernel(
    long long* __restrict__ Mq, long long ldm, double m_scale, int shift, int n, const EpilogueArgs ep) {
    constexpr int kWarps = kStructThreads / 32;
    constexpr int kCols = 32 * CPT;
    constexpr int kBatch = 8 / CPT;
    constexpr int kRowsPerWarp = kStructRows / kWarps;
    using Vec = StructVec<CPT>;
    __shared__ float4 s_fs[kStructRows];
    __shared__ double s_u[kStructRows];
    __shared__ float4 s_ft[kCols];
    __shared__ double s_v[kCols];
    __shared__ float2 cst[COLSTATS ? kWarps : 1][kCols];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int j0 = blockIdx.x * kCols;
    const int i0 = blockIdx.y * kStructRows;
    const int jb = j0 + CPT * lane;
    const bool has_f = ep.fs != nullptr;
    const bool has_d = !has_f && ep.D != nullptr;
    const float lam = static_cast<float>(ep.lam);
    const bool use_p = lam != 0.f;
    const double m_bias = -4503599627370496.0 * m_scale;
    for (int t = threadIdx.x; t < kStructRows; t += kStructThreads) {
        const int i = i0 + t;
        s_fs[t] = (has_f && i < n) ? reinterpret_cast<const float4*>(ep.fs)[i] : make_float4(0, 0, 0, 0);
        s_u[t] = (ep.U != nullptr && i < n) ? ep.U[i] : 0.0;
    }
    for (int t = threadIdx.x; t < kCols; t += kStructThreads) {
        const int j = j0 + t;
        s_ft[t] = (has_f && j < n) ? reinterpret_cast<const float4*>(ep.ft)[j] : make_float4(0, 0, 0, 0);
        s_v[t] = (ep.V != nullptr && j < n) ? ep.V[j] : 0.0;
    }
    __syncthreads();
    const bool full = jb + CPT - 1 < n;
    float cm[CPT], cs[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
        cm[c] = -INFINITY;
        cs[c] = 0.f;
    }
    const long long half = SHIFT ? (1ll << (shift - 1)) : 0;
    if (jb < n) {
        for (int r0 = 0; r0 < kRowsPerWarp; r0 += kBatch) {
            long long m[kBatch][CPT];
            float p[kBatch][CPT];
#pragma unroll
            for (int b = 0; b < kBatch; ++b) {
                const int i = i0 + warp + kWarps * (r0 + b);
#pragma unroll
                for (int c = 0; c < CPT; ++c) {
                    m[b][c] = 0;
                    p[b][c] = 0.f;
                }
                if (i >= n) continue;
                const long long* mrow = Mq + row_offset(i, ldm) + jb;
                const float* prow = ep.P + row_offset(i, ep.ldp) + jb;
                if (full) {
                    Vec::load_m(mrow, m[b]);
                    if (use_p) Vec::load_p(prow, p[b]);
                } else {
#pragma unroll
                    for (int c = 0; c < CPT; ++c) {
                        if (jb + c >= n) break;
                        m[b][c] = mrow[c];
                        if (use_p) p[b][c] = prow[c];
                    }
                }
            }
#pragma unroll
            for (int b = 0; b < kBatch; ++b) {
                const int ii = warp + kWarps * (r0 + b);
                const int i = i0 + ii;
                if (i >= n) break;
                const double ui = s_u[ii];
                const float4 f1 = s_fs[ii];
                float o[CPT];
#pragma unroll
                for (int c = 0; c < CPT; ++c) {
                    const float apb = fixed_to_float(m[b][c], m_scale, m_bias);
                    // the FP32 gradient in the order of gradient_kernel's scalar path
                    float reg = 0.f;
                    if (use_p) reg = __fmul_rn(lam, __fsub_rn(1.0f, __fmul_rn(2.0f, p[b][c])));
                    float g = __fadd_rn(__fmul_rn(-2.0f, apb), reg);
                    if (has_f) {
                        const float4 f2 = s_ft[CPT * lane + c];
                        const float d0 = __fsub_rn(f1.x, f2.x), d1 = __fsub_rn(f1.y, f2.y);
                        const float d2 = __fsub_rn(f1.z, f2.z), d3 = __fsub_rn(f1.w, f2.w);
                        const float ss = __fmaf_rn(d3, d3, __fmaf_rn(d2, d2, __fmaf_rn(d1, d1, __fmul_rn(d0, d0))));
                        float dist;
                        if constexpr (SQ) asm("sqrt.approx.f32 %0, %1;" : "=f"(dist) : "f"(ss));
                        else dist = __fsqrt_rn(ss);
                        g = __fadd_rn(g, dist);
                    } else if (has_d && jb + c < n) {
                        g = __fadd_rn(g, ep.D[row_offset(i, ep.ldd) + jb + c]);
                    }
                    o[c] = static_cast<float>(ep.out_scale * static_cast<double>(g) + (ui + s_v[CPT * lane + c]));
                    if (COLSTATS && (full || jb + c < n)) {
                        const float x = o[c] * kLog2e;
                        if (x > cm[c]) {
                            cs[c] = fmaf(cs[c], ex2(cm[c] - x), 1.0f);
                            cm[c] = x;
                        } else {
                            cs[c] += ex2(x - cm[c]);
                        }
                    }
                }
                float* orow = ep.out + row_offset(i, ep.ldo) + jb;
                long long* mrow = Mq + row_offset(i, ldm) + jb;
                if constexpr (SHIFT) {
#pragma unroll
                    for (int c = 0; c < CPT; ++c) m[b][c] = (m[b][c] + half) >> shift;
                }
                if (full) {
                    Vec::store_o(orow, o);
                    if constexpr (SHIFT) Vec::store_m(mrow, m[b]);
                } else {
#pragma unroll
                    for (int c = 0; c < CPT; ++c) {
                        if (jb + c >= n) break;
                        orow[c] = o[c];
                        if constexpr (SHIFT) mrow[c] = m[b][c];
                    }
                }
            }
        }
    }
    if constexpr (COLSTATS) {
#pragma unroll
        for (int c = 0; c < CPT; ++c) cst[warp][CPT * lane + c] = make_float2(cm[c], cs[c]);
        __syncthreads();
        if (threadIdx.x < kCols && j0 + static_cast<int>(threadIdx.x) < n) {
            const int t = threadIdx.x;
            float M = -INFINITY;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) M = fmaxf(M, cst[w][t].x);
            float S = 0.f;
            if (M != -INFINITY) {
#pragma unroll
                for (int w = 0; w < kWarps; ++w) {
                    const float2 ps = cst[w][t];
                    if (ps.x != -INFINITY) S += ps.y * ex2(ps.x - M);
                }
            }
            ep.colpart[static_cast<size_t>(blockIdx.y) * ep.ldc + j0 + t] = make_float2(M, S);
        }
    }
}

// out^T[j][i] = sign * sum_{k in N(i)} Q[j][k]  (M = Q^T operand of the reference's adjacency_matmul)
__global__ void spmm_transposed_operand_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                               const float* __restrict__ Q, long long ldq, int n,
                                               float* __restrict__ outT, long long ldo, float sign) {
    const int i = blockIdx.y * blockDim.x + threadIdx.x;
    const int j = blockIdx.x;
    if (i >= n) return;
    float acc = 0.f;
    const float* qrow = Q + static_cast<size_t>(j) * ldq;
    for (int e = rp[i]; e < rp[i + 1]; ++e) acc += qrow[col[e]];
    outT[static_cast<size_t>(j) * ldo + i] = sign * acc;
}

// Launch-shape knobs of the gradient kernels.  FUGAL_GATHER_UNROLL: gathers in
// flight per lane, 4 (default) or 8 (8 measured slower: 11.76 against 11.31 ms
// per step at n = 32768, the extra registers cost resident CTAs).
// FUGAL_GRAD_MIN_BLOCKS: resident CTAs per SM the epilogue kernel is compiled
// for, 8 (default: 32 registers with a few spills, 10.87 ms) or 6 (40 registers,
// no spills, 11.31 ms) -- the epilogue is issue-bound and needs the warps.
int gather_unroll() {
    const char* e = getenv("FUGAL_GATHER_UNROLL");
    return (e != nullptr && atoi(e) == 8) ? 8 : 4;
}
// The distance's square root: sqrt.approx by default, the rounding of the
// reference's distance kernel (built with --use_fast_math, cuda_kernels/setup.py:19);
// FUGAL_GRAD_SQRT_APPROX=0 takes the IEEE-rounded square root.
bool gradient_sqrt_approx() {
    const char* e = getenv("FUGAL_GRAD_SQRT_APPROX");
    return !(e != nullptr && atoi(e) == 0);
}
bool gradient_packed() {
    const char* e = getenv("FUGAL_GRAD_PACKED");
    return !(e != nullptr && atoi(e) == 0);
}
int gradient_min_blocks() {
    const char* e = getenv("FUGAL_GRAD_MIN_BLOCKS");
    return (e != nullptr && atoi(e) == 6) ? 6 : 8;
}

// col may be null for a graph without edges (it is never dereferenced then).
fugal_status check_csr(const int32_t* rp, const int32_t* col, int64_t n, const char* who) {
    (void)col;
    if (rp == nullptr) return fail(FUGAL_BAD_ARGUMENT, "%s: null row pointers", who);
    if (n <= 0 || n > (1ll << 30)) return fail(FUGAL_BAD_SHAPE, "%s: bad n", who);
    return FUGAL_OK;
}

}  // namespace fugal

using namespace fugal;

extern "C" fugal_status fugal_adjacency_matmul(const int32_t* col_indices, const int32_t* row_pointers, int64_t n,
                                               const float* M, int64_t ldm, int m_transposed, float* out,
                                               int64_t ldo, int negate, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    FUGAL_TRY(check_csr(row_pointers, col_indices, n, "fugal_adjacency_matmul"));
    if (M == nullptr || out == nullptr) return fail(FUGAL_BAD_ARGUMENT, "fugal_adjacency_matmul: null matrix");
    if (ldm < n || ldo < n) return fail(FUGAL_BAD_SHAPE, "fugal_adjacency_matmul: leading dimension < n");
    if (ldm >= (1ll << 32) || ldo >= (1ll << 32))
        return fail(FUGAL_BAD_SHAPE, "fugal_adjacency_matmul: leading dimension >= 2^32");
    const float sign = negate ? -1.f : 1.f;
    LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
    if (!m_transposed) {
        dim3 grid(static_cast<unsigned>((n + kTileRows - 1) / kTileRows),
                  static_cast<unsigned>((n + kTileCols - 1) / kTileCols));
        if ((ldm % 4) == 0 && aligned16(M))
            spmm_kernel<true><<<grid, kSpmmThreads, 0, stream>>>(row_pointers, col_indices, M, ldm,
                                                                  static_cast<int>(n), out, ldo, 0, sign);
        else
            spmm_kernel<false><<<grid, kSpmmThreads, 0, stream>>>(row_pointers, col_indices, M, ldm,
                                                                   static_cast<int>(n), out, ldo, 0, sign);
    } else {
        dim3 grid(static_cast<unsigned>(n), static_cast<unsigned>((n + 127) / 128));
        spmm_transposed_operand_kernel<<<grid, 128, 0, stream>>>(row_pointers, col_indices, M, ldm,
                                                                 static_cast<int>(n), out, ldo, sign);
    }
    return launch_check("fugal_adjacency_matmul");
}

extern "C" fugal_status fugal_gradient_workspace_size(int64_t n, size_t* bytes) {
    if (bytes == nullptr) return fail(FUGAL_BAD_ARGUMENT, "fugal_gradient_workspace_size: null output");
    if (n <= 0) return fail(FUGAL_BAD_SHAPE, "fugal_gradient_workspace_size: n must be positive");
    const int64_t ldt = (n + 3) / 4 * 4;
    *bytes = static_cast<size_t>(n) * ldt * sizeof(float);
    return FUGAL_OK;
}

namespace {

fugal_status fw_gradient(int64_t n, const int32_t* a_row_pointers, const int32_t* a_col_indices,
                         const int32_t* b_row_pointers, const int32_t* b_col_indices, const float* P, int64_t ldp,
                         const float* source_features, const float* target_features, const float* D, int64_t ldd,
                         double lambda, double lambda_scale, double out_scale, const double* U, const double* V,
                         float* out, int64_t ldo, void* workspace, size_t workspace_bytes, float* column_partials,
                         int64_t ldc, cudaStream_t stream) {
    FUGAL_TRY(check_csr(a_row_pointers, a_col_indices, n, "fugal_fw_gradient(A)"));
    FUGAL_TRY(check_csr(b_row_pointers, b_col_indices, n, "fugal_fw_gradient(B)"));
    if (P == nullptr || out == nullptr || workspace == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_fw_gradient: null pointer");
    if ((source_features == nullptr) != (target_features == nullptr))
        return fail(FUGAL_BAD_ARGUMENT, "fugal_fw_gradient: give both feature matrices or neither");
    if ((U == nullptr) != (V == nullptr)) return fail(FUGAL_BAD_ARGUMENT, "fugal_fw_gradient: give both U and V");
    if (source_features != nullptr && D != nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_fw_gradient: give features or a distance matrix, not both");
    if (D != nullptr && ldd < n) return fail(FUGAL_BAD_SHAPE, "fugal_fw_gradient: ldd < n");
    if (ldp < n || ldo < n || (ldp % 4) != 0 || !aligned16(P))
        return fail(FUGAL_BAD_SHAPE, "fugal_fw_gradient: P needs ld >= n, ld %% 4 == 0, 16-byte base");
    if (ldp >= (1ll << 32) || ldo >= (1ll << 32)) return fail(FUGAL_BAD_SHAPE, "fugal_fw_gradient: ld >= 2^32");
    if (source_features && (!aligned16(source_features) || !aligned16(target_features)))
        return fail(FUGAL_BAD_SHAPE, "fugal_fw_gradient: feature rows must be 16-byte aligned");
    if (column_partials != nullptr && (ldc < n || (reinterpret_cast<uintptr_t>(column_partials) & 7u) != 0))
        return fail(FUGAL_BAD_SHAPE, "fugal_fw_gradient_column_stats: partials need ldc >= n and 8-byte alignment");
    size_t need = 0;
    FUGAL_TRY(fugal_gradient_workspace_size(n, &need));
    if (workspace_bytes < need || !aligned16(workspace))
        return fail(FUGAL_WORKSPACE_TOO_SMALL, "fugal_fw_gradient: workspace %zu < %zu bytes", workspace_bytes, need);
    float* Tt = static_cast<float*>(workspace);
    const int64_t ldt = (n + 3) / 4 * 4;
    dim3 grid(static_cast<unsigned>((n + kTileRows - 1) / kTileRows),
              static_cast<unsigned>((n + kTileCols - 1) / kTileCols));
    const int unroll = gather_unroll();
    const int minb = gradient_min_blocks();
    {
        LaunchScope scope(FUGAL_KERNEL_GRADIENT, stream);
        if (unroll == 8)
            spmm_kernel<true, 8><<<grid, kSpmmThreads, 0, stream>>>(a_row_pointers, a_col_indices, P, ldp,
                                                                     static_cast<int>(n), Tt, ldt, 1, 1.f);
        else
            spmm_kernel<true, 4><<<grid, kSpmmThreads, 0, stream>>>(a_row_pointers, a_col_indices, P, ldp,
                                                                     static_cast<int>(n), Tt, ldt, 1, 1.f);
        FUGAL_TRY(launch_check("fugal_fw_gradient: A P"));
    }
    EpilogueArgs ep{P,   ldp, source_features, target_features, D, ldd, lambda * lambda_scale, out_scale, U, V, out,
                    ldo, reinterpret_cast<float2*>(column_partials), ldc};
    {
        LaunchScope scope(FUGAL_KERNEL_GRADIENT, stream);
        const int ni = static_cast<int>(n);
        const int* brp = b_row_pointers;
        const int* bci = b_col_indices;
        if (column_partials != nullptr) {
            if (unroll == 8 && minb == 8)
                gradient_kernel<true, 8, 8><<<grid, kSpmmThreads, 0, stream>>>(brp, bci, Tt, ldt, ni, ep);
            else if (unroll == 8)
                gradient_kernel<true, 8, 6><<<grid, kSpmmThreads, 0, stream>>>(brp, bci, Tt, ldt, ni, ep);
            else if (minb == 8 && !gradient_packed())
                gradient_kernel<true, 4, 8, false><<<grid, kSpmmThreads, 0, stream>>>(brp, bci, Tt, ldt, ni, ep);
            else if (minb == 8 && gradient_sqrt_approx())
                gradient_kernel<true, 4, 8, true, true><<<grid, kSpmmThreads, 0, stream>>>(brp, bci, Tt, ldt, ni, ep);
            else if (minb == 8)
                gradient_kernel<true, 4, 8><<<grid, kSpmmThreads, 0, stream>>>(brp, bci, Tt, ldt, ni, ep);
            else
                gradient_kernel<true, 4, 6><<<grid, kSpmmThreads, 0, stream>>>(brp, bci, Tt, ldt, ni, ep);
        } else {
            if (gradient_sqrt_approx())
                gradient_kernel<false, 4, 8, true, true><<<grid, kSpmmThreads, 0, stream>>>(brp, bci, Tt, ldt, ni, ep);
            else
                gradient_kernel<false, 4, 8><<<grid, kSpmmThreads, 0, stream>>>(brp, bci, Tt, ldt, ni, ep);
        }
        FUGAL_TRY(launch_check("fugal_fw_gradient: (A P) B + epilogue"));
    }
    return FUGAL_OK;
}

}  // namespace

extern "C" fugal_status fugal_fw_gradient(int64_t n, const int32_t* a_row_pointers, const int32_t* a_col_indices,
                                          const int32_t* b_row_pointers, const int32_t* b_col_indices,
                                          const float* P, int64_t ldp, const float* source_features,
                                          const float* target_features, const float* D, int64_t ldd,
                                          double lambda, double lambda_scale, double out_scale, const double* U,
                                          const double* V, float* out, int64_t ldo, void* workspace,
                                          size_t workspace_bytes, fugal_stream_t stream) {
    return fw_gradient(n, a_row_pointers, a_col_indices, b_row_pointers, b_col_indices, P, ldp, source_features,
                       target_features, D, ldd, lambda, lambda_scale, out_scale, U, V, out, ldo, workspace,
                       workspace_bytes, nullptr, 0, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" fugal_status fugal_gradient_column_chunks(int64_t n, int32_t* chunks) {
    if (chunks == nullptr) return fail(FUGAL_BAD_ARGUMENT, "fugal_gradient_column_chunks: null output");
    if (n <= 0 || n > (1ll << 30)) return fail(FUGAL_BAD_SHAPE, "fugal_gradient_column_chunks: bad n");
    *chunks = static_cast<int32_t>((n + kTileCols - 1) / kTileCols);
    return FUGAL_OK;
}

extern "C" fugal_status fugal_fw_gradient_column_stats(
    int64_t n, const int32_t* a_row_pointers, const int32_t* a_col_indices, const int32_t* b_row_pointers,
    const int32_t* b_col_indices, const float* P, int64_t ldp, const float* source_features,
    const float* target_features, const float* D, int64_t ldd, double lambda, double lambda_scale, double out_scale,
    const double* U, const double* V, float* out, int64_t ldo, void* workspace, size_t workspace_bytes,
    float* column_partials, int64_t ldc, fugal_stream_t stream) {
    if (column_partials == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_fw_gradient_column_stats: null column partials");
    return fw_gradient(n, a_row_pointers, a_col_indices, b_row_pointers, b_col_indices, P, ldp, source_features,
                       target_features, D, ldd, lambda, lambda_scale, out_scale, U, V, out, ldo, workspace,
                       workspace_bytes, column_partials, ldc, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" fugal_status fugal_structural_refresh(int64_t n, const int32_t* a_row_pointers,
                                                 const int32_t* a_col_indices, const int32_t* b_row_pointers,
                                                 const int32_t* b_col_indices, const float* P, int64_t ldp,
                                                 int64_t* Mq, int64_t ldm, int32_t frac_bits, void* workspace,
                                                 size_t workspace_bytes, int32_t* flags, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    const char* who = "fugal_structural_refresh";
    FUGAL_TRY(check_csr(a_row_pointers, a_col_indices, n, who));
    FUGAL_TRY(check_csr(b_row_pointers, b_col_indices, n, who));
    if (P == nullptr || Mq == nullptr || workspace == nullptr || flags == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "%s: null pointer", who);
    if (ldp < n || (ldp % 4) != 0 || !aligned16(P) || ldm < n || ldp >= (1ll << 32) || ldm >= (1ll << 32))
        return fail(FUGAL_BAD_SHAPE, "%s: P needs ld >= n, ld %% 4 == 0, 16-byte base; ldm >= n; ld < 2^32", who);
    if (frac_bits < 0 || frac_bits > 60) return fail(FUGAL_BAD_ARGUMENT, "%s: frac_bits must be in [0, 60]", who);
    size_t need = 0;
    FUGAL_TRY(fugal_gradient_workspace_size(n, &need));
    if (workspace_bytes < need || !aligned16(workspace))
        return fail(FUGAL_WORKSPACE_TOO_SMALL, "%s: workspace %zu < %zu bytes", who, workspace_bytes, need);
    float* Tt = static_cast<float*>(workspace);
    const int64_t ldt = (n + 3) / 4 * 4;
    dim3 grid(static_cast<unsigned>((n + kTileRows - 1) / kTileRows),
              static_cast<unsigned>((n + kTileCols - 1) / kTileCols));
    LaunchScope scope(FUGAL_KERNEL_GRADIENT, stream);
    spmm_kernel<true, 4><<<grid, kSpmmThreads, 0, stream>>>(a_row_pointers, a_col_indices, P, ldp,
                                                             static_cast<int>(n), Tt, ldt, 1, 1.f);
    FUGAL_TRY(launch_check("fugal_structural_refresh: A P"));
    structural_refresh_kernel<4><<<grid, kSpmmThreads, 0, stream>>>(b_row_pointers, b_col_indices, Tt, ldt,
                                                                     static_cast<int>(n),
                                                                     reinterpret_cast<long long*>(Mq), ldm,
                                                                     std::ldexp(1.0, frac_bits), flags);
    return launch_check("fugal_structural_refresh: (A P) B");
}

extern "C" fugal_status fugal_fw_gradient_structural(int64_t n, int64_t* Mq_, int64_t ldm, double m_scale,
                                                     int32_t shift, const float* P, int64_t ldp,
                                                     const float* source_features, const float* target_features,
                                                     const float* D, int64_t ldd, double lambda, double lambda_scale,
                                                     double out_scale, const double* U, const double* V, float* out,
                                                     int64_t ldo, float* column_partials, int64_t ldc,
                                                     fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    const char* who = "fugal_fw_gradient_structural";
    if (n <= 0 || n > (1ll << 30)) return fail(FUGAL_BAD_SHAPE, "%s: bad n", who);
    if (Mq_ == nullptr || P == nullptr || out == nullptr) return fail(FUGAL_BAD_ARGUMENT, "%s: null pointer", who);
    if ((source_features == nullptr) != (target_features == nullptr))
        return fail(FUGAL_BAD_ARGUMENT, "%s: give both feature matrices or neither", who);
    if ((U == nullptr) != (V == nullptr)) return fail(FUGAL_BAD_ARGUMENT, "%s: give both U and V", who);
    if (source_features != nullptr && D != nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "%s: give features or a distance matrix, not both", who);
    if (D != nullptr && ldd < n) return fail(FUGAL_BAD_SHAPE, "%s: ldd < n", who);
    if (ldm < n || (ldm % 4) != 0 || !aligned16(Mq_))
        return fail(FUGAL_BAD_SHAPE, "%s: Mq needs ld >= n, ld %% 4 == 0, 16-byte base", who);
    if (ldp < n || (ldp % 4) != 0 || !aligned16(P) || ldo < n || (ldo % 4) != 0 || !aligned16(out))
        return fail(FUGAL_BAD_SHAPE, "%s: P and out need ld >= n, ld %% 4 == 0, 16-byte base", who);
    if (ldp >= (1ll << 32) || ldo >= (1ll << 32) || ldm >= (1ll << 32) || (D != nullptr && ldd >= (1ll << 32)))
        return fail(FUGAL_BAD_SHAPE, "%s: ld >= 2^32", who);
    if (source_features && (!aligned16(source_features) || !aligned16(target_features)))
        return fail(FUGAL_BAD_SHAPE, "%s: feature rows must be 16-byte aligned", who);
    if (column_partials != nullptr && (ldc < n || (reinterpret_cast<uintptr_t>(column_partials) & 7u) != 0))
        return fail(FUGAL_BAD_SHAPE, "%s: partials need ldc >= n and 8-byte alignment", who);
    if (shift < 0 || shift > 62) return fail(FUGAL_BAD_ARGUMENT, "%s: shift must be in [0, 62]", who);
    EpilogueArgs ep{P,   ldp, source_features, target_features, D, ldd, lambda * lambda_scale, out_scale, U, V, out,
                    ldo, reinterpret_cast<float2*>(column_partials), ldc};
    const int cols = 32 * kStructCpt;
    dim3 grid(static_cast<unsigned>((n + cols - 1) / cols), static_cast<unsigned>((n + kStructRows - 1) / kStructRows));
    const int ni = static_cast<int>(n);
    long long* Mq = reinterpret_cast<long long*>(Mq_);
    LaunchScope scope(FUGAL_KERNEL_GRADIENT, stream);
    const bool sq = gradient_sqrt_approx();
    auto launch = [&](auto colstats, auto shifted, auto approx) {
        constexpr bool C = decltype(colstats)::value, S = decltype(shifted)::value, Q = decltype(approx)::value;
        gradient_structural_kernel<C, S, Q, kStructCpt>
            <<<grid, kStructThreads, 0, stream>>>(Mq, ldm, m_scale, shift, ni, ep);
    };
    using T = std::true_type;
    using F = std::false_type;
    const bool cp = column_partials != nullptr, sh = shift > 0;
    if (cp && sh) { if (sq) launch(T{}, T{}, T{}); else launch(T{}, T{}, F{}); }
    else if (cp)  { if (sq) launch(T{}, F{}, T{}); else launch(T{}, F{}, F{}); }
    else if (sh)  { if (sq) launch(F{}, T{}, T{}); else launch(F{}, T{}, F{}); }
    else          { if (sq) launch(F{}, F{}, T{}); else launch(F{}, F{}, F{}); }
    return launch_check(who);
}
