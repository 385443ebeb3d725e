// Entry points whose kernels land in convection.cu / particles.cu.
#include "ssg_internal.h"

using namespace ssg;

extern "C" {

ssg_status ssg_setup_dealias(ssg_context* c, int, const double*, const double*,
                             const double*, const double*, const double*) {
  return fail(c, SSG_ERR_STATE, "dealiasing set-up not available in this build");
}

ssg_status ssg_setup_particle_geometry(ssg_context* c, const double*, const double*) {
  return fail(c, SSG_ERR_STATE, "particle geometry set-up not available in this build");
}

ssg_status ssg_convection_operator(ssg_context* c, const double*, const double*, double*) {
  return fail(c, SSG_ERR_STATE, "convection not available in this build");
}

ssg_status ssg_set_particle_velocity(ssg_context* c, const double*) {
  return fail(c, SSG_ERR_STATE, "particles not available in this build");
}

ssg_status ssg_integrate_particle_equations(ssg_context* c, size_t, double*, int*, double,
                                            double, int*) {
  return fail(c, SSG_ERR_STATE, "particles not available in this build");
}

}
