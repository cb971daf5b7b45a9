// physics.h -- the Q-compensated physics imaging mode (panels + table lookup).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "internal.h"
#include "qpsdm_engine.h"

namespace qpsdm {

struct PhysicsState;

// One batch of records imaged into every line of the brick.  Per-line arrays
// are laid out line after line with the given strides (elements).
struct PhysicsBatch {
  const uint8_t *d_rec;
  int rec_bytes, ntr, big_endian, nlines;
  int *d_ints;
  size_t ints_ls;
  float *d_geom;
  size_t geom_ls;
  const float *d_taper200;
  const float *d_dips;  // line stride 4 * nxz
  size_t nxz;
  float *d_img;
  size_t img_ls;
  unsigned long long *d_npt;
  unsigned *d_err;
  KernelProfiler *prof;
  unsigned long long line_mask;  // bit il: line il of the brick takes this batch
};

// Line il of a brick takes the batch (lines past 64 always do).
inline bool batch_line_on(const PhysicsBatch &b, int il) {
  return il >= 64 || ((b.line_mask >> il) & 1ull);
}

int physics_create(PhysicsState **out, const qpsdm_static_params &p, std::string *err);
void physics_destroy(PhysicsState *s);
int physics_set_lines(PhysicsState *s, const qpsdm_static_params &p,
                      const qpsdm_line_params *lines, int nlines, cudaStream_t st,
                      std::string *err);
int physics_begin_offset(PhysicsState *s, const qpsdm_static_params &p,
                         const qpsdm_offset_params &o, int nlines, cudaStream_t st,
                         std::string *err);
int physics_process(PhysicsState *s, const qpsdm_static_params &p,
                    const qpsdm_line_params *lines, const qpsdm_offset_params &o,
                    const PhysicsBatch &b, cudaStream_t st, std::string *err);
int physics_tuning(const PhysicsState *s, int *variant, int *tz, int *tx, int *mb,
                   float *times, int ntimes);
// Panels of the last batch ([max_batch][nbins][nffti], the panel type) and,
// for FP16 panels, the per-trace sample multipliers.
void physics_panels(const PhysicsState *s, void **d_panels, float **d_pscale);
int physics_finalize_image(PhysicsState *s, float *d_img, size_t n, cudaStream_t st,
                           std::string *err);

}  // namespace qpsdm
