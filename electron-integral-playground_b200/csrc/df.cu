// Density-fitting contractions over the packed (mu nu|P) blocks of a batch:
//   gamma_P   = sum_{mu nu} (mu nu|P) D_{mu nu}
//   J_{mu nu} = sum_P (mu nu|P) c_P
// (the consumer of the integrals; the reference stops at the dense tensor,
// so this has no counterpart there).  Each class block of molecule m is a
// row-major matrix B[row][col], row = (pair shell, I, J), col = (K, aux shell):
//   B[((pair * n_i + I) * n_j + J)][K * n_aux + a]
// with the pair's first functions (i0, j0) in the batch's device pair table
// and the auxiliary shell's first function in its ket table.  Only shell pairs
// with i0 <= j0 are stored; an off-diagonal pair stands for (mu nu) and
// (nu mu), so gamma takes D_{mu nu} + D_{nu mu} and J gets the value at both
// (mu, nu) and (nu, mu).
//
// Both kernels stream every block once (the contractions are bound by HBM:
// 8 bytes read per integral, one FMA each).  Work items are (block, chunk of
// kDfRows rows).  gamma: the chunk's D weights are gathered into shared
// memory, each thread sums one column over the chunk's rows (coalesced reads
// along the row) and adds its column total into gamma with one atomic.  J:
// c is first gathered into each (molecule, auxiliary class)'s column order
// once (a small kernel); then each warp reduces four consecutive rows at a
// time against that contiguous, L2-resident vector (lanes along the rows, one
// load of c per column for the four) and adds the row totals into J with
// atomics (the blocks of the auxiliary classes of one pair class add into the
// same J elements).
#include "eip_common.cuh"
#include "eip_internal.h"

namespace eip {

constexpr int kDfThreads = 256;
constexpr int kDfRows = 32;
constexpr int kDfRowsPerWarp = 4;  // J: rows a warp reduces together (kDfRows = 8 warps x 4)

__device__ __forceinline__ int df_block_of(const DfBlock* __restrict__ blocks, int n_blocks, int item) {
    int lo = 0, hi = n_blocks - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (blocks[mid].item0 <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(kDfThreads)
df_gamma_kernel(const DfBlock* __restrict__ blocks, int n_blocks, int total_items, const double* __restrict__ packed,
                const double* __restrict__ D, double* __restrict__ gamma) {
    __shared__ double sx[kDfRows];
    for (int item = blockIdx.x; item < total_items; item += gridDim.x) {
        const DfBlock bk = blocks[df_block_of(blocks, n_blocks, item)];
        const int nij = bk.ni * bk.nj;
        const long long rows = (long long)bk.nsp * nij;
        const long long r0 = (long long)(item - bk.item0) * kDfRows;
        const int nr = (int)min((long long)kDfRows, rows - r0);
        const int cols = bk.nk * bk.nax;
        __syncthreads();  // sx of the previous item is no longer read
        if (threadIdx.x < nr) {
            const long long r = r0 + threadIdx.x;
            const int sp = (int)(r / nij), ij = (int)(r - (long long)sp * nij);
            const int I = ij / bk.nj, J = ij - I * bk.nj;
            const int2 ao = bk.ao[sp];
            const double* Dm = D + bk.d_off;
            const size_t mu = (size_t)ao.x + I, nu = (size_t)ao.y + J;
            double x = Dm[mu * bk.n_ao + nu];
            if (ao.x != ao.y) x += Dm[nu * bk.n_ao + mu];
            sx[threadIdx.x] = x;
        }
        __syncthreads();
        const double* B = packed + bk.out_off + r0 * cols;
        for (int col = threadIdx.x; col < cols; col += kDfThreads) {
            double acc = 0.0;
            for (int r = 0; r < nr; r++) acc = fma(sx[r], __ldg(B + (size_t)r * cols + col), acc);
            const int K = col / bk.nax, a = col - K * bk.nax;
            atomicAdd(gamma + bk.g_off + __ldg(bk.aux_start + a) + K, acc);
        }
    }
}

__global__ void df_gather_kernel(const DfGather* __restrict__ gathers, int n_gathers, long long total,
                                 const double* __restrict__ c, double* __restrict__ cg) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = n_gathers - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (gathers[mid].elem0 <= e) lo = mid;
            else hi = mid - 1;
        }
        const DfGather gt = gathers[lo];
        const int local = (int)(e - gt.elem0);
        const int K = local / gt.nax, a = local - K * gt.nax;
        cg[gt.cg_off + local] = c[gt.g_off + __ldg(gt.aux_start + a) + K];
    }
}

__global__ void __launch_bounds__(kDfThreads)
df_coulomb_kernel(const DfBlock* __restrict__ blocks, int n_blocks, int total_items,
                  const double* __restrict__ packed, const double* __restrict__ cg, double* __restrict__ Jout) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int kWarps = kDfThreads / 32;
    for (int item = blockIdx.x; item < total_items; item += gridDim.x) {
        const DfBlock bk = blocks[df_block_of(blocks, n_blocks, item)];
        const int nij = bk.ni * bk.nj;
        const long long rows = (long long)bk.nsp * nij;
        const long long r0 = (long long)(item - bk.item0) * kDfRows;
        const int nr = (int)min((long long)kDfRows, rows - r0);
        const int cols = bk.nk * bk.nax;
        const double* cm = cg + bk.cg_off;
        // each warp takes kDfRowsPerWarp consecutive rows at once: one load of
        // c per column feeds every row, and the rows' loads are in flight together
        for (int rr = warp * kDfRowsPerWarp; rr < nr; rr += kWarps * kDfRowsPerWarp) {
            const long long r = r0 + rr;
            const double* B = packed + bk.out_off + r * cols;
            const int nq = min(kDfRowsPerWarp, nr - rr);
            double s[kDfRowsPerWarp];
#pragma unroll
            for (int q = 0; q < kDfRowsPerWarp; q++) s[q] = 0.0;
            for (int col = lane; col < cols; col += 32) {
                const double cv = __ldg(cm + col);
#pragma unroll
                for (int q = 0; q < kDfRowsPerWarp; q++)
                    if (q < nq) s[q] = fma(__ldg(B + (size_t)q * cols + col), cv, s[q]);
            }
#pragma unroll
            for (int q = 0; q < kDfRowsPerWarp; q++)
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) s[q] += __shfl_xor_sync(0xffffffffu, s[q], o);
            // lane q adds row q into J (and its mirror)
            double mine = 0.0;
#pragma unroll
            for (int q = 0; q < kDfRowsPerWarp; q++)
                if (lane == q) mine = s[q];
            if (lane < nq) {
                const long long rq = r + lane;
                const int sp = (int)(rq / nij), ij = (int)(rq - (long long)sp * nij);
                const int I = ij / bk.nj, J = ij - I * bk.nj;
                const int2 ao = bk.ao[sp];
                double* Jm = Jout + bk.d_off;
                const size_t mu = (size_t)ao.x + I, nu = (size_t)ao.y + J;
                atomicAdd(Jm + mu * bk.n_ao + nu, mine);
                if (ao.x != ao.y) atomicAdd(Jm + nu * bk.n_ao + mu, mine);
            }
        }
    }
}

static int df_grid(int total_items) {
    int sms = 0;
    const int dev = current_device();
    if (dev < 0 || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    const int grid = 8 * sms;  // 8 CTAs of 256 threads per SM
    return total_items < grid ? total_items : grid;
}

int df_rows_per_item() { return kDfRows; }

int launch_df_gamma(const DfBlock* blocks, int n_blocks, int total_items, const double* packed, const double* D,
                    double* gamma, cudaStream_t s) {
    if (total_items <= 0 || n_blocks <= 0) return 0;
    const int grid = df_grid(total_items);
    if (grid <= 0) return 2;
    df_gamma_kernel<<<grid, kDfThreads, 0, s>>>(blocks, n_blocks, total_items, packed, D, gamma);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int launch_df_coulomb(const DfBlock* blocks, int n_blocks, int total_items, const DfGather* gathers, int n_gathers,
                      long long gather_elems, double* cg, const double* packed, const double* c, double* J,
                      cudaStream_t s) {
    if (total_items <= 0 || n_blocks <= 0) return 0;
    const int grid = df_grid(total_items);
    if (grid <= 0) return 2;
    if (gather_elems > 0) {
        const long long gb = (gather_elems + 255) / 256;
        df_gather_kernel<<<(unsigned)(gb < 148 * 16 ? gb : 148 * 16), 256, 0, s>>>(gathers, n_gathers, gather_elems, c,
                                                                                  cg);
        if (cudaGetLastError() != cudaSuccess) return 2;
    }
    df_coulomb_kernel<<<grid, kDfThreads, 0, s>>>(blocks, n_blocks, total_items, packed, cg, J);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

}  // namespace eip
