// Host-side declarations shared by the kernel translation units and the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace eip {

struct BraTable;
struct KetTable;
struct BatchMap;

int upload_constant_tables();
int upload_generic_tables();
const double* boys_table_device();
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

int generic_kc_chunk(int li, int lj, int lk);
size_t generic_smem_bytes(int li, int lj, int lk, int kc_chunk);
int launch_generic_raw(int mode, int li, int lj, int lk, const BraTable& bra, const KetTable& ket, double omega,
                       int skip_lower, double* raw, cudaStream_t s);
int launch_overlap_raw(int li, int lj, const BraTable& bra, const double* prim_b, double* raw, cudaStream_t s);
int launch_transform(int li, int lj, int lk, bool spherical, int n_bra, int n_ket, const double* raw, double* out,
                     cudaStream_t s);

}  // namespace eip
