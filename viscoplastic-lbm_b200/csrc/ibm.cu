// ibm.cu -- immersed-boundary step for movable spheres.
#include <cuda_runtime.h>
#include "sim.h"

namespace vlbm {

struct IbmState {
    int dummy_unused = 0;
};

vlbm_status ibm_step(vlbm_sim*) { return VLBM_OK; }
vlbm_status ibm_macroscopics_fixup(vlbm_sim*, float*, float*, float*, float*) { return VLBM_OK; }
void ibm_destroy(IbmState* st) { delete st; }
void ibm_reset(vlbm_sim*) {}

}  // namespace vlbm

using namespace vlbm;

extern "C" {

vlbm_status vlbm_ibm_config_default(vlbm_ibm_config* c) {
    if (!c) return VLBM_ERR_INVALID;
    *c = vlbm_ibm_config{};
    c->max_iterations = 1;       // ibmVar.h:23 IBM_MAX_ITERATION
    c->stencil = 4;              // ibmVar.h:136 STENCIL_4
    c->thickness = 1.0;          // ibmVar.h:33 IBM_THICKNESS
    c->movement_alpha = 0.5;     // ibmVar.h:95 IBM_MOVEMENT_DISCRETIZATION
    c->fluid_density = 1.0;      // ibmVar.h:110 FLUID_DENSITY
    c->gx = 0.0; c->gy = 0.0; c->gz = -5e-5;  // ibmVar.h:113-115
    c->wall_x = 0; c->wall_y = 1; c->wall_z = 0;  // ibmBoundaryCondition.h:20-56
    c->pp_friction = 0.1; c->pw_friction = 0.1;   // ibmBoundaryCondition.h:85-86
    c->pp_restitution = 0.9; c->pw_restitution = 0.9;  // ibmBoundaryCondition.h:87-88
    c->particle_young = 0.5; c->particle_poisson = 0.3;  // ibmBoundaryCondition.h:93-94
    c->wall_young = 100.0; c->wall_poisson = 0.3;        // ibmBoundaryCondition.h:97-98
    c->mesh_scale = 1.0;         // ibmVar.h:29 MESH_SCALE
    c->breugem = 0.0;            // ibmVar.h:27 BREUGEM_PARAMETER
    return VLBM_OK;
}

vlbm_status vlbm_add_spheres(vlbm_sim*, const vlbm_ibm_config*, const vlbm_sphere*, int32_t) {
    set_last_error("IBM spheres are not available in this build");
    return VLBM_ERR_UNSUPPORTED;
}

}  // extern "C"
