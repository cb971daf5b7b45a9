// physics.h -- the Q-compensated physics imaging mode (panels + table lookup).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "internal.h"
#include "qpsdm_engine.h"

namespace qpsdm {

struct PhysicsState;

struct PhysicsBatch {
  const uint8_t *d_rec;
  int rec_bytes, ntr, big_endian;
  int *d_ints;
  float *d_geom;
  const float *d_taper200;
  const float *d_dips;
  size_t nxz;
  float *d_img;
  unsigned long long *d_npt;
  unsigned *d_err;
  KernelProfiler *prof;
};

int physics_create(PhysicsState **out, const qpsdm_static_params &p, std::string *err);
void physics_destroy(PhysicsState *s);
int physics_set_line(PhysicsState *s, const qpsdm_static_params &p,
                     const qpsdm_line_params &l, cudaStream_t st, std::string *err);
int physics_begin_offset(PhysicsState *s, const qpsdm_static_params &p,
                         const qpsdm_offset_params &o, cudaStream_t st, std::string *err);
int physics_process(PhysicsState *s, const qpsdm_static_params &p,
                    const qpsdm_line_params &l, const qpsdm_offset_params &o,
                    const PhysicsBatch &b, cudaStream_t st, std::string *err);
int physics_finalize_image(PhysicsState *s, float *d_img, size_t n, cudaStream_t st,
                           std::string *err);

}  // namespace qpsdm
