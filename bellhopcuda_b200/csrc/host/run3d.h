// 3-D (BELLHOP3D) runner behind the C ABI: a batch of 3-D environments,
// their device tables, the trace / influence / scale sequence and the field
// access. A context holds either 2-D or 3-D environments.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../../include/bhcb.h"

namespace bhcb {

struct Run3;

Run3 *run3_new();
void run3_free(Run3 *r);
void run3_clear(Run3 *r);
int run3_count(const Run3 *r);
// reads and validates <root>.env and its companion files as a 3-D run; returns the env index
int run3_add_env(Run3 *r, const std::string &root);
// builds the tables, traces every ray of every environment and evaluates the
// fields; fills the statistics; returns the tracer's error bits (0 = clean)
// mixed: TL contributions of Cartesian geometric beams in mixed precision (the
// trace stays FP64)
uint32_t run3_run(Run3 *r, cudaStream_t st, int sm_count, uint64_t max_memory, int32_t opt_max_narr,
                  int32_t allow_merging, bool mixed, bhcb_stats &stats, uint32_t &warn_bits);
// arrivals runs (RunType 'A' / 'a'): storage [cell][max_narr], cells in the field layout
bool run3_is_arrivals(const Run3 *r);
// eigen-hit runs ('E'): copies up to max_hits hits of env (reference order) to
// hits (EigenHitRec records, may be NULL); returns their number
int64_t run3_eigen_hits(Run3 *r, int env, void *hits, int64_t max_hits);
int32_t run3_max_narr(const Run3 *r);
void run3_copy_arrivals(Run3 *r, int env, int32_t *narr, size_t narr_bytes, void *arr, size_t arr_bytes,
                        cudaStream_t st);
// dims = {nsz, nsx, nsy, ntheta, nrz, nrr}
void run3_shape(const Run3 *r, int env, int32_t dims[6]);
void run3_copy_field(Run3 *r, int env, void *dst, size_t bytes, cudaStream_t st);
void *run3_field_device(Run3 *r, int env);
// receiver grid and source positions as the reference's Position (m, deg)
void run3_grid(const Run3 *r, int env, std::vector<double> &sx, std::vector<double> &sy, std::vector<float> &sz,
               std::vector<double> &rr, std::vector<float> &rz, std::vector<double> &theta);
// ray runs ('R') and eigen runs ('E'): the traced (resp. re-traced hit) rays of
// env: per ray the point count, bounces of the last point, take-off
// declination (deg); the points (x, y, z) ray after ray
bool run3_has_rays(const Run3 *r);
void run3_rays_shape(Run3 *r, int env, cudaStream_t st, int64_t &nrays, int64_t &npoints);
void run3_copy_rays(Run3 *r, int env, cudaStream_t st, int32_t *npts, int32_t *bounces, double *alpha_deg,
                    double *xyz, size_t xyz_bytes);
// <root>.shd (TL), <root>.arr (arrivals) or <root>.ray (rays, eigenrays) in the reference's 3-D layouts
void run3_writeout(Run3 *r, int env, const std::string &root, cudaStream_t st);
std::vector<std::string> run3_warnings(const Run3 *r, int env);

} // namespace bhcb
