// physics.cu -- physics imaging mode (placeholder until the panel kernels land).
#include "physics.h"

namespace qpsdm {

struct PhysicsState {};

int physics_create(PhysicsState **out, const qpsdm_static_params &, std::string *err) {
  *out = nullptr;
  if (err) *err = "physics mode not built yet";
  return QPSDM_ENOTSUP;
}
void physics_destroy(PhysicsState *s) { delete s; }
int physics_set_line(PhysicsState *, const qpsdm_static_params &, const qpsdm_line_params &,
                     cudaStream_t, std::string *) { return QPSDM_ENOTSUP; }
int physics_begin_offset(PhysicsState *, const qpsdm_static_params &, const qpsdm_offset_params &,
                         cudaStream_t, std::string *) { return QPSDM_ENOTSUP; }
int physics_process(PhysicsState *, const qpsdm_static_params &, const qpsdm_line_params &,
                    const qpsdm_offset_params &, const PhysicsBatch &, cudaStream_t,
                    std::string *) { return QPSDM_ENOTSUP; }
int physics_finalize_image(PhysicsState *, float *, size_t, cudaStream_t, std::string *) {
  return QPSDM_ENOTSUP;
}

}  // namespace qpsdm
