// Kernels of the batched form: many independent products C_i = A_i * B_i run
// as one product of block-diagonal operands (see spgemm_batch_* in spgemm.cu).
#include "cta.cuh"
#include "kernels.hpp"

namespace b200 {
namespace {

constexpr int kBatchThreads = 256;

// NIP of every product i: sum over its rows r in [row_off[i], row_off[i+1])
// of A of sum_{k in A(r,:)} len(B(k,:)).  One CTA per product.
__global__ __launch_bounds__(kBatchThreads) void k_product_nip(
    const int32_t* __restrict__ a_rpt, const int32_t* __restrict__ a_col,
    const int32_t* __restrict__ b_rpt, const int32_t* __restrict__ row_off,
    long long* __restrict__ nip) {
    __shared__ long long s_part[kBatchThreads / kWarp];
    const int i = blockIdx.x;
    const int r0 = row_off[i];
    const int r1 = row_off[i + 1];
    const int e0 = a_rpt[r0];
    const int e1 = a_rpt[r1];
    long long s = 0;
    for (int e = e0 + threadIdx.x; e < e1; e += kBatchThreads) {
        const int c = __ldg(a_col + e);
        s += __ldg(b_rpt + c + 1) - __ldg(b_rpt + c);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long t = 0;
        for (int w = 0; w < kBatchThreads / kWarp; w++) t += s_part[w];
        nip[i] = t;
    }
}

// Split a group's C into per-product CSR: for product i (rows [r0, r1) of the
// group's C, local row 0 at r0), write its own row pointer starting at 0 into
// rpt_out + out_off[i] and shift its columns back to local indices.
__global__ __launch_bounds__(kBatchThreads) void k_unpack(
    const int32_t* __restrict__ c_rpt, int32_t* __restrict__ c_col,
    const int32_t* __restrict__ row_off, const int32_t* __restrict__ col_off,
    const int64_t* __restrict__ out_off, int32_t first, int32_t* __restrict__ rpt_out,
    int32_t* __restrict__ pos_out) {
    const int i = first + blockIdx.x;  // product index in the batch
    const int base_row = row_off[first];
    const int r0 = row_off[i] - base_row;
    const int r1 = row_off[i + 1] - base_row;
    const int p0 = c_rpt[r0];
    const int p1 = c_rpt[r1];
    if (threadIdx.x == 0) {
        pos_out[2 * i] = p0;
        pos_out[2 * i + 1] = p1 - p0;
    }
    int32_t* out = rpt_out + out_off[i];
    for (int t = threadIdx.x; t <= r1 - r0; t += kBatchThreads) out[t] = c_rpt[r0 + t] - p0;
    const int shift = col_off[i];
    for (int p = p0 + threadIdx.x; p < p1; p += kBatchThreads) c_col[p] -= shift;
}

// NIP of many independent pairs (A_i, B_i) in one launch: pair i's A entries
// are cut into chunks of kNipChunk, one CTA per chunk (cta_off[i] is pair i's
// first CTA); each CTA sums len(B_i(k,:)) over its entries and adds the total
// to nip[i] (zeroed by the caller) with one atomic.
constexpr int kNipChunk = 16384;

__global__ __launch_bounds__(kBatchThreads) void k_pairs_nip(const NipPair* __restrict__ pairs,
                                                            const int32_t* __restrict__ cta_off,
                                                            int32_t count,
                                                            long long* __restrict__ nip) {
    __shared__ long long s_part[kBatchThreads / kWarp];
    const int b = blockIdx.x;
    // the pair this CTA belongs to: the last i with cta_off[i] <= b
    int lo = 0;
    int hi = count;  // cta_off[count] > b
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (cta_off[mid] <= b) lo = mid;
        else hi = mid;
    }
    const NipPair pr = pairs[lo];
    const int e0 = (b - cta_off[lo]) * kNipChunk;
    const int e1 = min(e0 + kNipChunk, pr.nnz);
    long long s = 0;
    for (int e = e0 + threadIdx.x; e < e1; e += kBatchThreads) {
        const int c = __ldg(pr.a_col + e);
        s += __ldg(pr.b_rpt + c + 1) - __ldg(pr.b_rpt + c);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long t = 0;
        for (int w = 0; w < kBatchThreads / kWarp; w++) t += s_part[w];
        atomicAdd(reinterpret_cast<unsigned long long*>(nip + lo),
                  static_cast<unsigned long long>(t));
    }
}

}  // namespace

int32_t pairs_nip_ctas(int32_t nnz) { return (nnz + kNipChunk - 1) / kNipChunk; }

cudaError_t launch_pairs_nip(const NipPair* pairs, const int32_t* cta_off, int32_t count,
                             int32_t ctas, long long* nip, cudaStream_t s) {
    if (ctas <= 0) return cudaSuccess;
    k_pairs_nip<<<ctas, kBatchThreads, 0, s>>>(pairs, cta_off, count, nip);
    return cudaGetLastError();
}

cudaError_t launch_product_nip(const int32_t* a_rpt, const int32_t* a_col, const int32_t* b_rpt,
                               const int32_t* row_off, int32_t count, long long* nip,
                               cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    k_product_nip<<<count, kBatchThreads, 0, s>>>(a_rpt, a_col, b_rpt, row_off, nip);
    return cudaGetLastError();
}

cudaError_t launch_unpack(const int32_t* c_rpt, int32_t* c_col, const int32_t* row_off,
                          const int32_t* col_off, const int64_t* out_off, int32_t first,
                          int32_t count, int32_t* rpt_out, int32_t* pos_out, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    k_unpack<<<count, kBatchThreads, 0, s>>>(c_rpt, c_col, row_off, col_off, out_off, first,
                                             rpt_out, pos_out);
    return cudaGetLastError();
}

}  // namespace b200
