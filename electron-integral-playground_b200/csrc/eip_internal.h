// Host-side declarations shared by the kernel translation units and the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include <atomic>

#include "eip_common.cuh"  // BraTable, KetTable, BatchMap (held by value below)

namespace eip {


// Per-device state.  Every device this process uses gets its own copy of the
// constant tables (module data is per device), its own Boys-grid address and
// its own launch attributes; everything is keyed by the device current on the
// calling thread and set up once, under a lock, by the first use on it.
constexpr int kMaxDevices = 64;
// Current device of the calling thread, or -1 (no device / out of range).
int current_device();
// Uploads the constant tables to the current device once (thread-safe);
// returns 0 or a cudaError_t value.
int ensure_device_tables();
int upload_generic_tables();
// Device address of the Boys grid on the current device (sets the device up
// on first use); nullptr if that failed.
const double* boys_table_device();
// Occupancy-sized persistent grid of one kernel on the current device: the
// kernel's dynamic shared-memory limit is raised to smem_bytes and the
// per-device result is cached in *cache (an array of kMaxDevices entries,
// 0 = not yet computed).  Returns the grid size, or 0 on failure.
int persistent_grid(const void* kernel, int threads, size_t smem_bytes, std::atomic<int>* cache);
// Records the calling thread's last error (eip_last_error) and prints it:
// "<what>: <CUDA error string>", or "<what>" alone for cudaSuccess.
void set_error(const char* what, cudaError_t e);
int launch_boys_probe(int L, const double* dT, int n, double* dout, cudaStream_t s);

bool fast3c_supported(int li, int lj, int lk);
int fast3c_variant(int li, int lj, int lk);
int fast3c_set_variant(int li, int lj, int lk, int v);
int fast3c_variant_fp32(int li, int lj, int lk);
int fast3c_set_variant_fp32(int li, int lj, int lk, int v);
size_t e_table_doubles(int li, int lj);
int launch_e_table(int li, int lj, const BraTable& bra, double* prim_E, cudaStream_t s);
int launch_fast_point(int li, int lj, const BraTable& bra, const KetTable& ket, const BatchMap& map,
                      int total_items, double omega, double* out, int* counter, cudaStream_t s);
int launch_fast3c(int li, int lj, int lk, const BraTable& bra, const KetTable& ket, const BatchMap& map,
                  int total_items, double omega, double* out, int* counter, cudaStream_t s, bool fp32 = false);

// General kernel (k_generic.cu): any class, run-time angular momenta, over a
// work list whose items are (shell pair, auxiliary shell or charge, chunk of
// ket components); molecule m has n_pair * n_aux * general_chunks(...) items
// numbered from map.item_begin[m], FP64.  point: the ket is unit point charges
// (lk ignored).  counter[0] must be 0 at launch; counter[1] receives a status.
// Returns 0, 1 (unsupported class), 2 (CUDA failure) or 3 (too large).
int general_chunks(int li, int lj, int lk, bool point, bool spherical);
// Relative work of one item of a class (ordering items heaviest first).
double general_item_cost(int li, int lj, int lk, bool point, bool spherical);
// E tables of pair class (li, lj) for the general kernel (GenClassSpec::etab):
// general_e_doubles(li, lj) doubles per primitive pair of the bra table.
int general_e_doubles(int li, int lj);
int launch_general_e_table(int li, int lj, const BraTable& bra, int n_prim, double* out, cudaStream_t s);
// Entries of one item's Cartesian accumulator block (the partial block that a
// split item writes).
int general_block_entries(int li, int lj, int lk, bool point, bool spherical);
// One class of a multi-class general launch: its n_items items are numbered
// after the previous classes' (or come from perm); status: its self-check word.
// n_splits > 1: every block (x chunk of ket components) is n_splits
// consecutive items, each over its share of the block's units; they write
// partial blocks to partial[item * general_block_entries()] and the last to
// arrive (arrive[item / n_splits], 0 at launch and left 0) adds them in split
// order and stores the block.  Molecule m then has
// n_pair * n_aux * general_chunks() * n_splits items.
struct GenClassSpec {
    int li, lj, lk;
    bool point;
    BraTable bra;
    KetTable ket;
    BatchMap map;
    int n_items;
    int* status;
    int n_splits = 1;
    double* partial = nullptr;
    int* arrive = nullptr;
    const double* etab = nullptr;  // E tables per primitive pair, or nullptr (computed in the kernel)
};
int general_max_classes();
// Up to general_max_classes() classes in one persistent launch; perm (optional, device) lists
// (class, item within class) in the order the CTAs take them; counter[0]
// must be 0 at launch.  Returns 0, 1 (unsupported class), 2 or 3 (too large).
int launch_general_multi(const GenClassSpec* specs, int n, bool spherical, const int2* perm, double omega,
                         double* out, int* counter, cudaStream_t s);
int launch_general(int li, int lj, int lk, bool point, bool spherical, const BraTable& bra, const KetTable& ket,
                   const BatchMap& map, int total_items, double omega, double* out, int* counter, cudaStream_t s);
// One packed class block of one molecule as a density-fitting matrix (df.cu):
// rows (pair shell, I, J), columns (K, auxiliary shell).
struct DfBlock {
    long long out_off;     // first element in the packed buffer
    long long d_off;       // the molecule's D / J offset (n_ao^2 doubles per molecule)
    long long g_off;       // the molecule's gamma / c offset (n_aux doubles per molecule)
    const int2* ao;        // the block's shell pairs: first functions (i0, j0), device
    const int* aux_start;  // the block's auxiliary shells: first function, device
    long long cg_off;      // the block's (molecule, auxiliary class) gathered c vector
    int nsp, ni, nj, nk, nax, n_ao;
    int item0;             // first work item of the block (df_rows_per_item() rows each)
};
// One (molecule, auxiliary class) column vector of the J contraction:
// cg[cg_off + K * nax + a] = c[g_off + aux_start[a] + K].
struct DfGather {
    long long cg_off, g_off;
    const int* aux_start;
    int nk, nax;
    long long elem0;  // first element of this vector in the launch
};
int df_rows_per_item();
// gamma += sum (mu nu|P) D and J += sum (mu nu|P) c over every block (device pointers).
int launch_df_gamma(const DfBlock* blocks, int n_blocks, int total_items, const double* packed, const double* D,
                    double* gamma, cudaStream_t s);
// J: first the c vectors are gathered into each block's column order (cg),
// then every block row is reduced against its gathered vector.
int launch_df_coulomb(const DfBlock* blocks, int n_blocks, int total_items, const DfGather* gathers, int n_gathers,
                      long long gather_elems, double* cg, const double* packed, const double* c, double* J,
                      cudaStream_t s);
int launch_overlap_raw(int li, int lj, const BraTable& bra, const double* prim_b, double* raw, cudaStream_t s);
int launch_transform(int li, int lj, int lk, bool spherical, int n_bra, int n_ket, const double* raw, double* out,
                     cudaStream_t s);

}  // namespace eip
