// Kernel declarations shared by the step orchestration (driver.cu) and the kernel files.
#pragma once

#include "device.cuh"

namespace mdelast {

// scalar-kernel modes
enum PostMode : int { POST_INIT = 0, POST_STEP = 1 };

__global__ void k_cell_bin(AtomsView A);
__global__ void k_cell_sort(AtomsView A);
__global__ void k_nbr_build(AtomsView A, int cells_done);
__global__ void k_nbr_cells(AtomsView A);
size_t nbr_cells_smem(int cell_cap); // dynamic shared memory of k_nbr_cells
constexpr int kCellSortWarps = 8;      // half cells per k_cell_sort block (one warp each)
constexpr int kNbrCellsThreads = 256;   // threads of a k_nbr_cells block (one 2x2x2 half-cell group)
constexpr size_t kNbrCellsStaticSmem = 4 * 1024; // bound on k_nbr_cells' static shared memory
// launchers of the templated pair kernels (defined beside them); tpa = lanes per atom,
// one of 1, 4, 8, 16 (valid_tpa)
bool valid_tpa(int tpa);
void launch_density(bool obs, int tpa, int grid, cudaStream_t s, AtomsView const &A,
                    TablesView const &T);
void launch_force(bool obs, bool kick, int tpa, int grid, cudaStream_t s, AtomsView const &A,
                  TablesView const &T);
// the same passes with FP32 pair math (mixed precision)
void launch_density_mx(bool obs, int tpa, int grid, cudaStream_t s, AtomsView const &A,
                       TablesView const &T);
void launch_force_mx(bool obs, bool kick, int tpa, int grid, cudaStream_t s, AtomsView const &A,
                     TablesView const &T);
// the mixed force pass with the quintic tables staged in shared memory (T.st_n > 0; tpa 4,
// 8 or 16; blocks of kStagedBlock threads); prepare_force_mx_staged raises the kernels'
// dynamic shared-memory limit (to the staging budget) before any launch or capture
constexpr int kStagedBlock = 512;
void launch_force_mx_staged(bool obs, bool kick, int tpa, int grid, cudaStream_t s,
                            AtomsView const &A, TablesView const &T);
cudaError_t prepare_force_mx_staged(int smem_bytes);
__global__ void k_posf(AtomsView A);
__global__ void k_kick_drift(AtomsView A, TablesView T);
__global__ void k_pre(AtomsView A);
__global__ void k_reduce(AtomsView A);
__global__ void k_post(AtomsView A, int mode, int obs);
__global__ void k_samples_reset(AtomsView A, int what);
__global__ void k_sublist(AtomsView A);
// k_sublist's dynamic shared memory for rows of capacity maxn (0: rows keep list order)
constexpr size_t kSublistSortMax = 96 * 1024;
__host__ __device__ size_t sublist_smem(int maxn);
__global__ void k_sub_invalidate(AtomsView A);
__global__ void k_readout(AtomsView A, TablesView T, int r, int field, double *out,
                          const double *pos0, int stepped);
__global__ void k_half_list_counts(AtomsView A, int r, int *counts);
__global__ void k_half_list_fill(AtomsView A, int r, const int *point, int *out);
__global__ void k_status_and(AtomsView A, unsigned mask);
__global__ void k_table_eval(TablesView T, int which, int s, const double *x, int n,
                             double *out);

} // namespace mdelast
