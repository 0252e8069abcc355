// Graph structure kernels: CSR construction and the four FUGAL node features.
//   fugal_create_adjacency            cuda_kernels/adjacency.cu:163-259 (CUB sort + row pointers)
//   fugal_graph_features              cuda_kernels/feature_extraction.cu:13-84
//   fugal_average_neighbor_features   cuda_kernels/feature_extraction.cu:86-125
//
// Triangle counts are integer and exact: t(v) = sum over u in N(v) of
// |N(v) & N(u)|, one warp per vertex with lanes over the neighbours and a
// binary search of the shorter sorted list in the longer one (a hub's list is
// searched, never merged element by element by a single thread, so BA hubs do
// not serialise a warp).  The clustering ratio uses the IEEE-rounded FP32
// division.  Neighbour averages keep the reference's sequential FP32 sum in CSR
// order (one thread per vertex), so they are bit-reproducible.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>

#include "fugal_common.cuh"
#include "fugal_host.h"

namespace fugal {

__device__ __forceinline__ int lower_bound(const int* __restrict__ col, int lo, int hi, int x) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (col[mid] < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__global__ void graph_features_kernel(const int* __restrict__ col, const int* __restrict__ rp, int n,
                                      float* clustering, float* degrees, int* degree_counts, long long* tri_counts) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
        const int s = rp[v], e = rp[v + 1];
        const int d = e - s;
        long long t = 0;
        for (int idx = s + lane; idx < e; idx += 32) {
            const int u = col[idx];
            const int us = rp[u], ue = rp[u + 1];
            int as = s, ae = e, bs = us, be = ue;  // search the shorter list in the longer
            if (ue - us < e - s) {
                as = us; ae = ue; bs = s; be = e;
            }
            int cnt = 0;
            for (int k = as; k < ae; ++k) {
                const int x = col[k];
                const int pos = lower_bound(col, bs, be, x);
                cnt += (pos < be && col[pos] == x) ? 1 : 0;
            }
            t += cnt;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) {
            degrees[v] = static_cast<float>(d);
            if (degree_counts) degree_counts[v] = d;
            if (tri_counts) tri_counts[v] = t;
            const float denom = static_cast<float>(static_cast<long long>(d) * (d - 1));
            clustering[v] = (t == 0 || d < 2) ? 0.0f : __fdiv_rn(static_cast<float>(t), denom);
        }
    }
}

__global__ void average_neighbor_kernel(const int* __restrict__ col, const int* __restrict__ rp, int n,
                                        const float* __restrict__ f, float* avg) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int s = rp[v], e = rp[v + 1];
        float sum = 0.0f;
        for (int k = s; k < e; ++k) sum = __fadd_rn(sum, f[col[k]]);
        const int d = e - s;
        avg[v] = d == 0 ? 0.0f : __fdiv_rn(sum, static_cast<float>(d));
    }
}

// ---------------------------------------------------------------- CSR build

__global__ void count_rows_kernel(const int* edges, long long m, int n, int* counts, int* bad) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m; e += (long long)gridDim.x * blockDim.x) {
        const int x = edges[2 * e], y = edges[2 * e + 1];
        if (x < 0 || x >= n || y < 0 || y >= n) {
            atomicExch(bad, 1);
            continue;
        }
        atomicAdd(&counts[y], 1);
    }
}

// Exclusive scan of counts[0..n) into rp[0..n] by one block (carry across chunks).
__global__ void __launch_bounds__(1024) scan_rows_kernel(const int* counts, int n, int* rp, int* cursor) {
    __shared__ int warp_tot[32];
    __shared__ int carry_s;
    if (threadIdx.x == 0) carry_s = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int x = i < n ? counts[i] : 0;
        int incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            int w = lane < (blockDim.x >> 5) ? warp_tot[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            warp_tot[lane] = w;  // inclusive over warps
        }
        __syncthreads();
        const int carry = carry_s;
        const int excl = carry + (warp > 0 ? warp_tot[warp - 1] : 0) + incl - x;
        if (i < n) {
            rp[i] = excl;
            cursor[i] = excl;
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry_s = excl + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) rp[n] = carry_s;
}

__global__ void scatter_cols_kernel(const int* edges, long long m, int n, int* cursor, int* col) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m; e += (long long)gridDim.x * blockDim.x) {
        const int x = edges[2 * e], y = edges[2 * e + 1];
        if (x < 0 || x >= n || y < 0 || y >= n) continue;
        const int pos = atomicAdd(&cursor[y], 1);
        col[pos] = x;
    }
}

// Sort each row's columns ascending: bitonic sort in shared memory, one block
// per row, rows up to kMaxSortRow entries (longer rows raise a flag).
constexpr int kMaxSortRow = 8192;

__global__ void __launch_bounds__(512) sort_rows_kernel(const int* rp, int n, int* col, int* bad) {
    __shared__ int buf[kMaxSortRow];
    for (int r = blockIdx.x; r < n; r += gridDim.x) {
        const int s = rp[r], e = rp[r + 1], d = e - s;
        if (d <= 1) continue;
        if (d > kMaxSortRow) {
            if (threadIdx.x == 0) atomicExch(bad, 2);
            continue;
        }
        int size = 1;
        while (size < d) size <<= 1;
        for (int i = threadIdx.x; i < size; i += blockDim.x) buf[i] = i < d ? col[s + i] : INT_MAX;
        __syncthreads();
        for (int k = 2; k <= size; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = threadIdx.x; i < size; i += blockDim.x) {
                    const int ij = i ^ j;
                    if (ij > i) {
                        const bool up = (i & k) == 0;
                        const int a = buf[i], b = buf[ij];
                        if ((a > b) == up) {
                            buf[i] = b;
                            buf[ij] = a;
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (int i = threadIdx.x; i < d; i += blockDim.x) col[s + i] = buf[i];
        __syncthreads();
    }
}

}  // namespace fugal

using namespace fugal;

extern "C" fugal_status fugal_graph_features(const int32_t* col_indices, const int32_t* row_pointers, int64_t n,
                                             float* clustering, float* degrees, int32_t* degree_counts,
                                             int64_t* triangle_counts, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    if (row_pointers == nullptr || clustering == nullptr || degrees == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_graph_features: null argument");
    if (n <= 0 || n > INT_MAX - 1) return fail(FUGAL_BAD_SHAPE, "fugal_graph_features: bad n");
    const int threads = 256;
    const int blocks = static_cast<int>(std::min<int64_t>((n * 32 + threads - 1) / threads, 32 * sm_count()));
    LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
    graph_features_kernel<<<blocks, threads, 0, stream>>>(col_indices, row_pointers, static_cast<int>(n), clustering,
                                                          degrees, degree_counts,
                                                          reinterpret_cast<long long*>(triangle_counts));
    return launch_check("fugal_graph_features");
}

extern "C" fugal_status fugal_average_neighbor_features(const int32_t* col_indices, const int32_t* row_pointers,
                                                        int64_t n, const float* features, float* averages,
                                                        fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    if (row_pointers == nullptr || features == nullptr || averages == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_average_neighbor_features: null argument");
    if (n <= 0 || n > INT_MAX - 1) return fail(FUGAL_BAD_SHAPE, "fugal_average_neighbor_features: bad n");
    const int blocks = static_cast<int>(std::min<int64_t>((n + 127) / 128, 16 * sm_count()));
    LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
    average_neighbor_kernel<<<blocks, 128, 0, stream>>>(col_indices, row_pointers, static_cast<int>(n), features,
                                                        averages);
    return launch_check("fugal_average_neighbor_features");
}

extern "C" fugal_status fugal_create_adjacency_workspace_size(int64_t edge_count, int64_t node_count,
                                                              size_t* bytes) {
    if (bytes == nullptr) return fail(FUGAL_BAD_ARGUMENT, "fugal_create_adjacency_workspace_size: null output");
    if (edge_count < 0 || node_count <= 0 || node_count > INT_MAX - 1)
        return fail(FUGAL_BAD_SHAPE, "fugal_create_adjacency_workspace_size: bad sizes");
    // counts [n+1], cursor [n+1], flag word
    *bytes = static_cast<size_t>(2 * (node_count + 1) + 4) * sizeof(int);
    return FUGAL_OK;
}

extern "C" fugal_status fugal_create_adjacency(const int32_t* edges, int64_t edge_count, int64_t node_count,
                                               int32_t* col_indices, int32_t* row_pointers, void* workspace,
                                               size_t workspace_bytes, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    size_t need = 0;
    FUGAL_TRY(fugal_create_adjacency_workspace_size(edge_count, node_count, &need));
    if (row_pointers == nullptr || workspace == nullptr || (edge_count > 0 && (edges == nullptr || col_indices == nullptr)))
        return fail(FUGAL_BAD_ARGUMENT, "fugal_create_adjacency: null argument");
    if (workspace_bytes < need)
        return fail(FUGAL_WORKSPACE_TOO_SMALL, "fugal_create_adjacency: workspace %zu < %zu", workspace_bytes, need);
    const int n = static_cast<int>(node_count);
    int* counts = static_cast<int*>(workspace);
    int* cursor = counts + (n + 1);
    int* bad = cursor + (n + 1);
    FUGAL_TRY(cuda_check(cudaMemsetAsync(counts, 0, need, stream), "fugal_create_adjacency: clear"));
    const int blocks = static_cast<int>(std::min<int64_t>((edge_count + 255) / 256 + 1, 8 * sm_count()));
    {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        count_rows_kernel<<<blocks, 256, 0, stream>>>(edges, edge_count, n, counts, bad);
        FUGAL_TRY(launch_check("fugal_create_adjacency: count"));
    }
    {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        scan_rows_kernel<<<1, 1024, 0, stream>>>(counts, n, row_pointers, cursor);
        FUGAL_TRY(launch_check("fugal_create_adjacency: scan"));
    }
    if (edge_count > 0) {
        {
            LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
            scatter_cols_kernel<<<blocks, 256, 0, stream>>>(edges, edge_count, n, cursor, col_indices);
            FUGAL_TRY(launch_check("fugal_create_adjacency: scatter"));
        }
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        const int sblocks = static_cast<int>(std::min<int64_t>(n, 8 * sm_count()));
        sort_rows_kernel<<<sblocks, 512, 0, stream>>>(row_pointers, n, col_indices, bad);
        FUGAL_TRY(launch_check("fugal_create_adjacency: sort"));
    }
    return FUGAL_OK;
}
