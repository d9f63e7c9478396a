// Particle placement for the reference build of a sphere case (test infrastructure).
//
// ref_build.py compiles this file in place of IBM/ibmParticlesCreation.cpp,
// whose createParticles (ibmParticlesCreation.cpp:5-43) places the reference's
// demonstration ellipsoid.  Here every sphere of the case is meshed by the
// reference's own Particle::makeSpherePolar (IBM/structs/particle.cpp:698), the
// call createParticles keeps commented out for spheres, with MESH_COULOMB
// optimisation steps, movable, PARTICLE_DENSITY and at rest.
//
// REF_SPHERES is the list "d0, cx0, cy0, cz0, d1, cx1, ..." that ref_build.py
// writes into ref_spheres.h from the case's `spheres`.
#include "ibmParticlesCreation.h"
#include "ref_spheres.h"

#ifdef IBM

void createParticles(Particle* particles)
{
    static const double spec[] = {REF_SPHERES};
    static_assert(sizeof(spec) / sizeof(spec[0]) == 4 * NUM_PARTICLES,
                  "REF_SPHERES must hold diameter, cx, cy, cz per particle");
    for (int p = 0; p < NUM_PARTICLES; p++) {
        const double* s = spec + 4 * p;
        particles[p].makeSpherePolar((dfloat)s[0], dfloat3((dfloat)s[1], (dfloat)s[2], (dfloat)s[3]), MESH_COULOMB,
                                     true, PARTICLE_DENSITY, dfloat3(0, 0, 0), dfloat3(0, 0, 0));
    }
}

#endif  // IBM
