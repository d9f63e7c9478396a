/*
 * vlbm.h -- C ABI of the B200-native VISCOPLASTIC-LBM fluid time step.
 *
 * Plain C linkage, plain pointers and sizes, no CUDA or torch types in any
 * signature.  Every call returns a vlbm_status (0 = ok); nothing calls exit().
 * One simulation handle per host thread.  The library's only global state is
 * the per-device kernel caches and one fixed device array that
 * vlbm_moments_sum_noalloc uses as scratch (calls of it that overlap on a
 * device race; see its declaration).  Host buffers are owned by the caller,
 * device buffers by the library.
 *
 * The reference has no library boundary: its hot path is entered through
 * CUDA kernels and compile-time macros.  Each entry point below names the
 * reference interface it replaces (paths inside CERNN/VISCOPLASTIC-LBM).
 */
#ifndef VLBM_H
#define VLBM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VLBM_ABI_VERSION 2

typedef int vlbm_status;
enum {
    VLBM_OK = 0,
    VLBM_ERR_INVALID = 1,      /* bad argument or configuration           */
    VLBM_ERR_CUDA = 2,         /* CUDA runtime error (message: vlbm_last_error) */
    VLBM_ERR_NOMEM = 3,        /* device or host allocation failed        */
    VLBM_ERR_UNSUPPORTED = 4,  /* combination the reference does not define */
    VLBM_ERR_DIVERGED = 5,     /* non-finite or non-positive density seen  */
    VLBM_ERR_STATE = 6,        /* call out of order (e.g. no geometry yet) */
    /* 7 is not used */
    VLBM_ERR_NOT_FOUND = 8,    /* unknown name / missing file              */
    VLBM_ERR_IO = 9            /* host file I/O failed                     */
};

/* Velocity sets: src/CUDA/velocitySets/D3Q19.h:31-46, D3Q27.h:39-56. */
enum { VLBM_D3Q19 = 19, VLBM_D3Q27 = 27 };

/* Collision operator.  REGULARIZED is the operator compiled by default in
 * src/CUDA/lbm.cu:263-461; BGK is src/CUDA/collisionSchemes/collisionForceNoReg.txt. */
enum { VLBM_OP_REGULARIZED = 0, VLBM_OP_BGK = 1 };

/* Rheology: src/CUDA/NNF/nnf.h:10-24 (POWERLAW / BINGHAM), Newtonian otherwise. */
enum { VLBM_NEWTONIAN = 0, VLBM_BINGHAM = 1, VLBM_POWERLAW = 2 };

/* Population storage.  F32 is the reference's `dfloat=float` layout; F16/BF16
 * store scaled deviations (f_i - w_i*rho0)*scale, arithmetic stays FP32. */
enum { VLBM_STORE_F32 = 0, VLBM_STORE_F16 = 1, VLBM_STORE_BF16 = 2 };

/* Node-map bit layout, identical to src/CUDA/structs/nodeTypeMap.h:15-133 so a
 * map produced by a reference builder (gpuBuildBoundaryConditions) can be
 * passed unchanged to vlbm_set_node_map. */
#define VLBM_MAP_RHO_IDX_OFFSET 0
#define VLBM_MAP_UZ_IDX_OFFSET 3
#define VLBM_MAP_UY_IDX_OFFSET 6
#define VLBM_MAP_UX_IDX_OFFSET 9
#define VLBM_MAP_GEOMETRY_OFFSET 12
#define VLBM_MAP_DIRECTION_OFFSET 13
#define VLBM_MAP_SCHEME_OFFSET 18
#define VLBM_MAP_IS_USED_OFFSET 21
#define VLBM_MAP_SAVE_POST_COL_OFFSET 22
/* Interpolated bounce-back: unknown in-plane directions, bit d for the D2Q9
 * direction d of (1,0), (0,1), (-1,0), (0,-1), (1,1), (-1,1), (-1,-1), (1,-1)
 * (SPC_INTERP_BB_OFFSET, nodeTypeMap.h:98-107); the wall is the inner cylinder
 * when the direction field is VLBM_SOUTH, the outer one when VLBM_NORTH
 * (setIsInsideNodeInterpoBB, nodeTypeMap.h:306-319). */
#define VLBM_MAP_INTERP_BB_OFFSET 23

/* BC schemes (nodeTypeMap.h:35-56) */
enum {
    VLBM_BC_NULL = 0, VLBM_BC_VEL_ZOUHE = 1, VLBM_BC_VEL_BOUNCE_BACK = 2,
    VLBM_BC_PRES_ZOUHE = 3, VLBM_BC_FREE_SLIP = 4, VLBM_BC_BOUNCE_BACK = 5,
    VLBM_BC_INTERP_BOUNCE_BACK = 6, VLBM_BC_SPECIAL = 7
};
/* Directions (nodeTypeMap.h:59-85) */
enum {
    VLBM_NORTH = 0, VLBM_SOUTH = 1, VLBM_WEST = 2, VLBM_EAST = 3, VLBM_FRONT = 4, VLBM_BACK = 5,
    VLBM_NORTH_WEST = 6, VLBM_NORTH_EAST = 7, VLBM_NORTH_FRONT = 8, VLBM_NORTH_BACK = 9,
    VLBM_SOUTH_WEST = 10, VLBM_SOUTH_EAST = 11, VLBM_SOUTH_FRONT = 12, VLBM_SOUTH_BACK = 13,
    VLBM_WEST_FRONT = 14, VLBM_WEST_BACK = 15, VLBM_EAST_FRONT = 16, VLBM_EAST_BACK = 17,
    VLBM_NORTH_WEST_FRONT = 18, VLBM_NORTH_WEST_BACK = 19, VLBM_NORTH_EAST_FRONT = 20,
    VLBM_NORTH_EAST_BACK = 21, VLBM_SOUTH_WEST_FRONT = 22, VLBM_SOUTH_WEST_BACK = 23,
    VLBM_SOUTH_EAST_FRONT = 24, VLBM_SOUTH_EAST_BACK = 25
};
enum { VLBM_CONCAVE = 0, VLBM_CONVEX = 1 };

/* Named geometry builders (the builder .cu files of
 * src/CUDA/boundaryConditionsBuilders/ that the reference copies into src/CUDA/). */
enum {
    VLBM_BUILDER_PERIODIC = 0,          /* no boundary nodes                           */
    VLBM_BUILDER_PLATES_Y = 1,          /* parallelPlatesBounceBack_Y.cu: walls y=0, y=NY-1 */
    VLBM_BUILDER_LID_DRIVEN = 2,        /* lidDrivenBounceBack.cu: walls x,y, lid y=NY-1, z periodic */
    VLBM_BUILDER_CLOSED_BOX = 3,        /* closedBoxBounceBack.cu: all six faces       */
    VLBM_BUILDER_SQUARE_DUCT = 4,       /* squareDuctBounceBack.cu: walls x,y, z periodic */
    VLBM_BUILDER_DUCT_YZ = 5,           /* square duct walls y,z, periodic x (serving ducts) */
    VLBM_BUILDER_LID_CAVITY_CLOSED = 6, /* all six faces, moving lid at y=NY-1          */
    VLBM_BUILDER_PLATES_Y_FREE_SLIP = 7,/* bounce-back y=0, free-slip y=NY-1            */
    VLBM_BUILDER_PLATES_Y_ZOUHE = 8,    /* velocity Zou-He at y=0 and y=NY-1 (Couette)  */
    VLBM_BUILDER_CIRCULAR_DUCT = 9,     /* circularDuctInterpBounceBack.cu: cylinder along z,
                                           interpolated bounce-back, nodes outside unused */
    VLBM_BUILDER_ANNULAR_DUCT = 10      /* annularDuctInterpBounceBack.cu: outer and inner
                                           cylinders along z (INTERNAL_DUCT_BC)           */
};

typedef struct vlbm_config {
    int32_t nx, ny, nz;          /* lattice size (var.h:95-100: NX, NY, NZ_TOTAL)  */
    int32_t vel_set;             /* VLBM_D3Q19 / VLBM_D3Q27                         */
    int32_t collision;           /* VLBM_OP_*                                       */
    int32_t rheology;            /* VLBM_NEWTONIAN / BINGHAM / POWERLAW             */
    int32_t storage;             /* VLBM_STORE_*                                    */
    int32_t device;              /* CUDA device ordinal                             */
    double tau;                  /* var.h:104 TAU (Newtonian relaxation time)       */
    double rho0;                 /* var.h:107 RHO_0                                 */
    double fx, fy, fz;           /* var.h:109-111 body force FX, FY, FZ             */
    double eta_p;                /* nnf.h:20 ETA_P (Bingham plastic viscosity)      */
    double yield_stress;         /* nnf.h:21 S_Y                                    */
    double n_index;              /* nnf.h:11 N_INDEX (Power-Law)                    */
    double k_consistency;        /* nnf.h:12 K_CONSISTENCY                          */
    double gamma0;               /* nnf.h:13 GAMMA_0 (truncation)                   */
    double ux_bc[8], uy_bc[8], uz_bc[8], rho_bc[8]; /* var.h:114-117 UX_BC..RHO_BC */
    double storage_scale;        /* F16/BF16 deviation scale; 0 = library default (F16: a power of two 1..2^24) */
    int32_t layout;              /* VLBM_LAYOUT_*: population storage order          */
    /* z-slab of a larger lattice (one slab per GPU, lbm.cu:601-657 N_GPUS):
     * slab_nz_total > 0 is the whole lattice's NZ and global plane
     * slab_z_offset + z is this lattice's plane z (its first and last planes
     * being the ghost planes, see vlbm_halo_pack).  0, 0 for a whole lattice. */
    int32_t slab_z_offset, slab_nz_total;
    int32_t reserved[5];
    /* Cylindrical ducts (var.h:142-162), axis along z through the lattice centre
     * (DUCT_CENTER_X/Y).  Radii <= 0 take the var.h values: outer NY/2 - 1.5,
     * inner outer/4.  Wall motion of the interpolated bounce-back
     * (interpolatedBounceBack.cu:26-58): axial velocity and angular velocity of
     * each cylinder; the outer rotation is scaled by z/NZ as in the reference.
     * vlbm_set_builder uses these radii; vlbm_build_node_map (no configuration)
     * the var.h values. */
    double duct_outer_radius, duct_inner_radius;
    double duct_outer_velocity, duct_outer_rotation;
    double duct_inner_velocity, duct_inner_rotation;
} vlbm_config;

/* Population storage order.  NATURAL: planes [Q][z][y][x].  ZPAIR: nodes z and
 * z+NZ/2 of the same (x, y) are adjacent, so every stencil access of the fused
 * step is one aligned two-node vector (requires even NZ) and the arithmetic
 * runs on packed FP32x2.  AUTO picks ZPAIR for even NZ with FP16/BF16 storage
 * or D3Q27, NATURAL otherwise (D3Q19 FP32).  The layout is internal: every
 * entry point takes and returns the [z][y][x] order. */
enum { VLBM_LAYOUT_AUTO = 0, VLBM_LAYOUT_NATURAL = 1, VLBM_LAYOUT_ZPAIR = 2 };

/* Fill `cfg` with the reference defaults (var.h / nnf.h values, D3Q19, FP32,
 * regularized, Newtonian, tau=0.6, rho0=1, zero force, UX_BC etc. from var.h:114-117). */
vlbm_status vlbm_config_default(vlbm_config* cfg);

typedef struct vlbm_sim vlbm_sim;

/* Replaces the allocation + gpuInitialization sequence of src/CUDA/main.cu:114-216
 * (Populations::popAllocation populations.h:46-52, Macroscopics::macrAllocation
 * macroscopics.h:83-124, gpuInitialization lbmInitialization.cu:48-90).
 * Populations start at f_eq(rho0, u=0) (lbmInitialization.cu:93-111). */
vlbm_status vlbm_create(const vlbm_config* cfg, vlbm_sim** out);
vlbm_status vlbm_destroy(vlbm_sim* sim);

/* Replaces gpuBuildBoundaryConditions + setupBoundaryConditionsInfo
 * (main.cu:174-194, boundaryConditionsInfo.h:76-116): takes the per-node 32-bit
 * map in the reference's bit layout, [nz][ny][nx] order (idxScalar,
 * globalFunctions.h:111-115).  n must equal nx*ny*nz. */
vlbm_status vlbm_set_node_map(vlbm_sim* sim, const uint32_t* map, size_t n);
/* Same tables as vlbm_build_node_map(builder, ...) + vlbm_set_node_map, built
 * from the builder's rules on the domain faces only (no N-word map on the
 * host): the set-up cost scales with the lattice surface, not its volume. */
vlbm_status vlbm_set_builder(vlbm_sim* sim, int32_t builder);

/* Host-side restatement of the named builders; writes nx*ny*nz words. */
vlbm_status vlbm_build_node_map(int builder, int nx, int ny, int nz, uint32_t* map_out, size_t n);

/* Re-initialise populations to equilibrium at (rho, ux, uy, uz) everywhere and
 * reset step counter, omega state and IBM forces (lbmInitialization.cu:48-150). */
vlbm_status vlbm_init_equilibrium(vlbm_sim* sim, double rho, double ux, double uy, double uz);

/* Advance nsteps fluid time steps (one iteration of the loop at main.cu:270-394
 * each: gpuMacrCollisionStream lbm.cu:4-504, gpuPopulationsTransfer lbm.cu:601-657,
 * gpuApplyBC lbm.cu:580-598, and the IBM step ibm.cu:6-192 when spheres exist).
 * Asynchronous on the simulation's stream. */
vlbm_status vlbm_step(vlbm_sim* sim, uint32_t nsteps);

/* Block until the simulation's stream is idle; returns VLBM_ERR_DIVERGED when the
 * device-side guard saw a non-finite or non-positive density since the last check. */
vlbm_status vlbm_sync(vlbm_sim* sim);

/* Use an external CUDA stream (cudaStream_t passed as void*; NULL = library stream). */
vlbm_status vlbm_set_stream(vlbm_sim* sim, void* cuda_stream);

/* Macroscopics of the current state, the values gpuMacrCollisionStream would save
 * (lbm.cu:79-111, 247-261) and copyMacr would bring to the host
 * (macroscopics.h:173-283): rho, u = (sum f c + F/2)/rho, omega.  Host arrays of
 * nx*ny*nz floats in [nz][ny][nx] order; any pointer may be NULL.  With spheres
 * present the values are those after the IBM step (ibm.cu:544-648 plus the
 * multi-direct-forcing velocity corrections). */
vlbm_status vlbm_get_macroscopics(vlbm_sim* sim, float* rho, float* ux, float* uy,
                                  float* uz, float* omega);
/* Same into device pointers (each nx*ny*nz floats), asynchronous. */
vlbm_status vlbm_get_macroscopics_device(vlbm_sim* sim, float* rho, float* ux, float* uy,
                                         float* uz, float* omega);

/* Populations f_i(x) of the current state after boundary conditions, [Q][nz][ny][nx]
 * floats (idxPop order without the ghost plane, globalFunctions.h:143-147). */
vlbm_status vlbm_get_populations(vlbm_sim* sim, float* pops, size_t n);

/* Set the full population state (same layout); resets boundary side-state. */
vlbm_status vlbm_set_populations(vlbm_sim* sim, const float* pops, size_t n);

/* Global mass and momentum of the current state in FP64: out4 = {sum rho,
 * sum rho*ux, sum rho*uy, sum rho*uz} with rho*u = sum_i f_i c_i + F/2 per node
 * (host array of 4 doubles).  Replaces the FP32 density reduction of
 * AuxFunctions/reduction.cu:36-98 / auxFunction.cu:3-62 and the host sums of
 * treatData.cpp:25-449.  Allocates its partial-sum buffer on first use. */
vlbm_status vlbm_moments_sum(vlbm_sim* sim, double* out4);

/* Same sums as vlbm_moments_sum, for callers that cannot allocate device
 * memory when they need them (a serving process whose HBM is all committed to
 * admitted simulations, a monitor thread in a process whose allocator belongs
 * to another framework).  It allocates nothing: it uses a fixed 512 KiB scratch
 * array in the library's device globals, which every GPU that loads the
 * library keeps until exit.  No counterpart in the reference.  Limit: lattices
 * of at most 67,108,864 nodes (larger ones return VLBM_ERR_INVALID).  The
 * first call on a device looks up the array's device address, so make that
 * first call before any stream capture.  All calls on a device share the
 * array: calls that overlap on the GPU race, so serialise them.  out4 is a
 * host array of 4 doubles; results are bit-identical to vlbm_moments_sum. */
vlbm_status vlbm_moments_sum_noalloc(vlbm_sim* sim, double* out4);

/* Per-node IBM force (macr.f, macroscopics.h) of the current state, [3][nz][ny][nx]. */
vlbm_status vlbm_get_forces(vlbm_sim* sim, float* fxyz, size_t n);

typedef struct vlbm_info {
    int32_t nx, ny, nz, q;
    int32_t storage_bytes;       /* bytes per stored population value            */
    int64_t step;                /* current step counter                          */
    int64_t n_bc_nodes;          /* boundary nodes with side-state                */
    int64_t device_bytes;        /* device memory held by the simulation          */
    double bytes_per_node_step;  /* algorithmic bytes: 2*Q*storage_bytes          */
    int32_t n_particles, n_lagrangian_nodes;
    int32_t last_kernel_variant; /* autotuned launch variant of the fused kernel  */
    int32_t layout;              /* population layout in use: 0 natural, 1 z-paired,
                                    2 z-paired in blocks of 32 pair-nodes         */
    int32_t aa_parity;           /* 1: the next step is the in-place scheme's odd
                                    (neighbour) step, the one that needs halos  */
    int32_t reserved[5];
} vlbm_info;
vlbm_status vlbm_get_info(vlbm_sim* sim, vlbm_info* info);

/* ---------------------------------------------------------------- IBM --- */
/* IBM parameters (src/CUDA/IBM/ibmVar.h:21-126, ibmBoundaryCondition.h:19-107). */
typedef struct vlbm_ibm_config {
    int32_t max_iterations;      /* IBM_MAX_ITERATION                             */
    int32_t stencil;             /* 4 = Peskin 4-point (STENCIL_4), 2 = STENCIL_2  */
    double thickness;            /* IBM_THICKNESS                                  */
    double movement_alpha;       /* IBM_MOVEMENT_DISCRETIZATION                    */
    double fluid_density;        /* FLUID_DENSITY                                  */
    double gx, gy, gz;           /* GX, GY, GZ                                     */
    int32_t wall_x, wall_y, wall_z; /* 1 = IBM_BC_?_WALL, 0 = IBM_BC_?_PERIODIC    */
    double pp_friction, pw_friction, pp_restitution, pw_restitution;
    double particle_young, particle_poisson, wall_young, wall_poisson;
    double mesh_scale;           /* MESH_SCALE                                     */
    double breugem;              /* BREUGEM_PARAMETER                              */
    int32_t reserved[8];
} vlbm_ibm_config;

typedef struct vlbm_sphere {
    double diameter;
    double cx, cy, cz;
    double vx, vy, vz;
    double wx, wy, wz;
    double density;
    int32_t movable;
    int32_t reserved;
} vlbm_sphere;

/* Particle state, the ParticleCenter fields (IBM/structs/particleCenter.h:65-118)
 * that saveParticlesInfo writes (IBM/ibmReport.cpp:26-102). */
typedef struct vlbm_particle_state {
    double pos[3], vel[3], w[3], f[3], M[3];
    double pos_old[3], vel_old[3], w_old[3], f_old[3], M_old[3];
    double w_avg[3], w_pos[3];
    double I[6];                 /* xx, yy, zz, xy, xz, yz                        */
    double radius, volume, density, S;
    int32_t movable, n_nodes;
} vlbm_particle_state;

vlbm_status vlbm_ibm_config_default(vlbm_ibm_config* cfg);
/* Replaces createParticles (IBM/ibmParticlesCreation.cpp:5-43) with
 * Particle::makeSpherePolar (IBM/structs/particle.cpp:698-995) per sphere, and
 * ParticlesSoA::updateParticlesAsSoA (particle.cpp:5-62).  Call before vlbm_step. */
vlbm_status vlbm_add_spheres(vlbm_sim* sim, const vlbm_ibm_config* ibm,
                             const vlbm_sphere* spheres, int32_t n);
vlbm_status vlbm_get_particles(vlbm_sim* sim, vlbm_particle_state* out, int32_t n);
/* Lagrangian node positions [3][n_nodes] doubles and forces [3][n_nodes]. */
vlbm_status vlbm_get_lagrangian_nodes(vlbm_sim* sim, double* pos, double* force, size_t n_nodes);

/* ------------------------------------------------------------ outputs --- */
/* Write PATH/ID/ID_<var><step>.bin files (lbmReport.cpp:55-172) for rho, ux, uy,
 * uz [, fx, fy, fz when export_forces and spheres exist] [, omega when non-Newtonian].
 * The step field is getVarFilename's: six digits (ID_rho000100.bin), seven for
 * step 0 (ID_rho0000000.bin), the plain number from 1,000,000 on. */
vlbm_status vlbm_write_macr_bin(vlbm_sim* sim, const char* path_files, const char* id_sim,
                                uint32_t step_label, int32_t export_forces);
/* Write PATH/ID/ID_info.txt, the run-information file of saveSimInfo /
 * getSimInfoString (lbmReport.cpp:174-386): simulation, non-Newtonian, IBM and
 * CUDA sections with the reference's keys and number formats.  The caller
 * passes what the reference keeps in SimInfo and var.h: steps run, elapsed
 * seconds (MLUPS = steps * N / 1e6 / seconds), DATA_REPORT, MACR_SAVE and
 * U_MAX.  "Bandwidht" (sic, the reference's key) is this library's
 * algorithmic bytes per second in 2^30-byte units; F16/BF16 runs add a
 * "Population storage" line. */
vlbm_status vlbm_write_info(vlbm_sim* sim, const char* path_files, const char* id_sim, uint64_t total_steps,
                            double time_elapsed_s, int32_t report_steps, int32_t save_steps, double u_max);

/* Particle files of saveParticlesInfo (IBM/ibmReport.cpp:26-102):
 * PATH/ID/ID_pCenters<step>.csv (one row per sphere: p_number, step, pos, vel,
 * w, f, M, I, S, radius, volume, movable, semi-axes; %e numbers) and, when
 * save_nodes, PATH/ID/ID_pNodes<step>.csv (particle_index, pos, S per
 * Lagrangian node).  The step field is getVarFilename's, as for the .bin files.
 * VLBM_ERR_STATE when the simulation has no spheres. */
vlbm_status vlbm_write_particles_csv(vlbm_sim* sim, const char* path_files, const char* id_sim, uint32_t step_label,
                                     int32_t save_nodes);

/* ------------------------------------------------- run configuration --- */
/* The run configuration of the drop-in driver (driver/vlbm_run.cpp), read from
 * the YAML file of the reference's configuration tool: a list whose first item
 * maps the keys of pyvisc's SchemeVarH (pyvisc/schemes.py:53-74,
 * examples/all_options.yaml) -- precision, NX, NY, NZ (per GPU), tau, vel_set,
 * use_ibm, non_newtonian_model (null / BINGHAM / POWERLAW), sim_id, path_save,
 * steps, macr_save, data_report, FX, FY, FZ, data_stop, data_save, pop_save,
 * ini_step, n_gpus, resid_max -- with SchemeVarH's defaults and type checks.
 * Extension keys carry the other compile-time constants the reference keeps in
 * var.h, nnf.h and ibmVar.h: rho_0, u_max, ux_bc/uy_bc/uz_bc/rho_bc (lists),
 * collision (regularized / bgk), eta_p, yield_stress, n_index, k_consistency,
 * gamma_0, storage (f32 / f16 / bf16), device, builder (a VLBM_BUILDER_* name:
 * periodic, plates_y, lid_driven, closed_box (default, the builder compiled by
 * default), square_duct, duct_yz, lid_cavity_closed, plates_y_free_slip,
 * plates_y_zouhe, circular_duct, annular_duct), outer_radius, inner_radius,
 * outer_velocity, outer_rotation, inner_velocity, inner_rotation,
 * checkpoint_save, load_checkpoint, checkpoint_folder, and a mapping `ibm`
 * (max_iterations, stencil, thickness, movement_discretization, fluid_density,
 * gx, gy, gz, wall_x/y/z, pp/pw_friction, pp/pw_restitution, particle/wall
 * young and poisson, mesh_scale, breugem, particles_save, particles_nodes_save,
 * export_forces, particle_density, spheres: a list of {diameter, center: [x,y,z],
 * velocity, angular_velocity, density, movable}).  Other keys are ignored, as
 * pydantic ignores them.  precision: double and n_gpus > 1 return
 * VLBM_ERR_UNSUPPORTED; a malformed file or value VLBM_ERR_INVALID with the key
 * and line in vlbm_last_error. */
typedef struct vlbm_run_config {
    vlbm_config cfg;             /* lattice and physics                            */
    vlbm_ibm_config ibm;         /* IBM parameters (key `ibm`)                      */
    int32_t builder;             /* VLBM_BUILDER_*                                  */
    int32_t use_ibm;             /* use_ibm                                         */
    int32_t precision_double;    /* precision == "double" (rejected)                */
    int32_t n_gpus;              /* n_gpus (1)                                      */
    int64_t steps;               /* steps (N_STEPS)                                 */
    int64_t ini_step;            /* ini_step (INI_STEP)                             */
    int64_t macr_save;           /* macr_save (MACR_SAVE; 0 = off)                  */
    int64_t data_report;         /* data_report (DATA_REPORT; 0 = off)              */
    int64_t checkpoint_save;     /* CHECKPOINT_SAVE (0 = off)                       */
    int64_t particles_save;      /* IBM_PARTICLES_SAVE (0 = off)                    */
    int32_t data_stop, data_save, pop_save, load_checkpoint;
    int32_t particles_nodes_save;/* IBM_PARTICLES_NODES_SAVE                        */
    int32_t export_forces;       /* EXPORT_FORCES                                   */
    int32_t n_spheres;           /* entries under ibm.spheres                       */
    int32_t reserved0;
    double resid_max;            /* resid_max (RESID_MAX)                           */
    double u_max;                /* U_MAX                                           */
    char sim_id[32];             /* ID_SIM: sim_id as '%03d' (var.h.j2)              */
    char path_save[256];         /* PATH_FILES                                      */
    char load_folder[256];       /* SIMULATION_FOLDER_LOAD_CHECKPOINT               */
    int32_t reserved[16];
} vlbm_run_config;

/* Parse YAML text (or read the file at `path`) into `out`; the spheres listed
 * are written to `spheres` (up to max_spheres; out->n_spheres counts them all).
 * Replaces pyvisc's read_configs + render (pyvisc/conf_handler.py:15-24,
 * pyvisc/__main__.py:6-9) and the compile step. */
vlbm_status vlbm_run_config_parse(const char* yaml_text, vlbm_run_config* out, vlbm_sphere* spheres,
                                  int32_t max_spheres);
vlbm_status vlbm_run_config_load(const char* path, vlbm_run_config* out, vlbm_sphere* spheres,
                                 int32_t max_spheres);

/* --------------------------------------------------------- checkpoint --- */
/* Complete state of a simulation as one image (replaces operateSimCheckpoint /
 * saveSimCheckpoint / loadSimCheckpoint, simCheckpoint.cu:216-318, which write
 * and read step, pop, popAux, rho, u, omega, f and the IBM arrays as raw files):
 * populations as stored, boundary side stores, Power-Law omega, IBM force field
 * and node classes, device step counters, particle and Lagrangian-node state,
 * with a header that names the lattice, storage, layout and geometry and a
 * trailing hash.  A run resumed from an image continues bit for bit like the
 * run that wrote it.  Both calls synchronise the simulation's stream.
 *
 * vlbm_checkpoint_save: writes the image into `buf` (`n` bytes) and its size
 * into `*needed` (may be NULL); `buf` NULL only reports the size; a buffer
 * smaller than the image returns VLBM_ERR_INVALID with nothing written.
 * vlbm_checkpoint_load: the simulation must have been created with the same
 * nx, ny, nz, velocity set, storage (and scale) and layout, have the same
 * geometry and, with spheres, the same particle and node counts (the reference
 * creates its particles before loading them too); otherwise VLBM_ERR_INVALID
 * and the simulation is unchanged.  A corrupt or truncated image:
 * VLBM_ERR_INVALID; another format version: VLBM_ERR_UNSUPPORTED. */
vlbm_status vlbm_checkpoint_save(vlbm_sim* sim, void* buf, size_t n, size_t* needed);
vlbm_status vlbm_checkpoint_load(vlbm_sim* sim, const void* buf, size_t n);
/* The same image as the file PATH/ID/checkpoint/0_state.bin (the reference's
 * <gpu>_<name>.bin naming under PATH/ID/checkpoint; folders created as needed,
 * written to a temporary name and renamed).  Missing file: VLBM_ERR_NOT_FOUND. */
vlbm_status vlbm_save_checkpoint(vlbm_sim* sim, const char* path_files, const char* id_sim);
vlbm_status vlbm_load_checkpoint(vlbm_sim* sim, const char* path_files, const char* id_sim);

/* ----------------------------------------------------- data treatment --- */
/* Report-step data treatment on the device (treatData.cpp:25-89 and stopSim
 * treatData.cpp:451-460, which copy rho and u to the host and loop in FP32):
 *   residual = sum |u - u_prev| / sum |u| (1 when sum |u| = 0), u_prev = the
 *              velocity at the previous call (zero before the first call and
 *              after vlbm_init_equilibrium / vlbm_set_populations), the
 *              reference's macrCPUOld (main.cu:430-434);
 *   avg_rho  = sum rho / N;
 *   avg_uz_plane_xz[y] = sum over x, z of uz / (NX * NZ), when not NULL (`ny`
 *              must then be NY); the mean of this call, where the reference's
 *              avgUzPlanXZ keeps adding every report's mean (never cleared);
 *   stop     = residual < resid_max || avg_rho < 0 (RESID_MAX, var.h:119: 1e-5).
 * Sums are FP64 on the device in a fixed order (bit-reproducible); 3 + NY
 * doubles are copied to the host.  Synchronises the simulation's stream. */
typedef struct vlbm_treat {
    int64_t step;
    double residual;
    double avg_rho;
    int32_t stop;
    int32_t reserved;
} vlbm_treat;
vlbm_status vlbm_treat_data(vlbm_sim* sim, double resid_max, vlbm_treat* out, double* avg_uz_plane_xz,
                            int32_t ny);

/* ------------------------------------------------------------ serving --- */
typedef struct vlbm_server vlbm_server;
typedef struct vlbm_request {
    vlbm_config cfg;
    int32_t builder;             /* VLBM_BUILDER_*                                */
    uint32_t steps;              /* steps to run before completion                */
    uint64_t tag;                /* caller's id, returned in the completion      */
    int32_t n_spheres;
    const vlbm_sphere* spheres;  /* copied at submit                              */
    vlbm_ibm_config ibm;
} vlbm_request;
typedef struct vlbm_completion {
    uint64_t tag;
    vlbm_status status;
    double submit_time_s, start_time_s, finish_time_s; /* server clock, seconds   */
    double mean_ux;              /* volume-averaged ux of the final state         */
    uint64_t steps;
} vlbm_completion;

/* A continuous-batching server on one GPU: requests are admitted by HBM budget,
 * stay resident, advance together in one batched launch per step, and retire at
 * their step count.  A lattice is built without host waits on a high-priority
 * stream of its own (uploads from pinned staging); lattices with spheres or
 * large enough to fill a wave of the batched kernel step with launches of
 * their own in the library's layout.  The reference has no counterpart (one
 * compile-time simulation per process). */
vlbm_status vlbm_server_create(int device, size_t hbm_budget_bytes, int32_t max_resident,
                               vlbm_server** out);
vlbm_status vlbm_server_submit(vlbm_server* srv, const vlbm_request* req);
/* Advance every resident simulation by up to `steps` steps, admitting queued work
 * as memory frees up; returns the number of completions copied to `out`. */
vlbm_status vlbm_server_pump(vlbm_server* srv, uint32_t steps, vlbm_completion* out,
                             int32_t max_out, int32_t* n_out);
vlbm_status vlbm_server_stats(vlbm_server* srv, int32_t* resident, int32_t* queued,
                              int64_t* bytes_in_use, double* lattice_updates);
/* Copy the macroscopics of the finished request `tag` (kept until fetched). */
vlbm_status vlbm_server_fetch(vlbm_server* srv, uint64_t tag, float* ux, size_t n);
/* Counters since creation.  Host seconds in: [0] admission (building new
 * lattices), [1] table rebuilds, [2] enqueuing steps (graph captures
 * included), [3] waiting for the GPU (queue depth limit, idle read-outs),
 * [4] completing read-outs; then [5] batch steps, [6] kernels launched
 * directly, [7] graph launches, [8] graph captures, [9] host seconds in graph
 * captures (part of [2]); then the device bytes of the server's memory cache,
 * [10] held by resident and retiring lattices and [11] cached for reuse (their
 * sum stays within the HBM budget); then the parts of [0]: [12] creating
 * lattices, [13] their boundary tables, [14] their spheres, [15] handing
 * them to the server stream.  Writes min(n, 16) values. */
vlbm_status vlbm_server_profile(vlbm_server* srv, double* seconds, int32_t n);
/* Tuning: sphere-free lattices with at least `nodes` nodes get their own
 * single-lattice launch each step instead of sharing the batched launch.
 * -1 (the default): lattices that fill a wave of the batched kernel (148 SMs x
 * resident blocks x 256 nodes) get one, largest first, while the estimated
 * host launch time of a step stays below 60 % of its estimated GPU time. */
vlbm_status vlbm_server_set_own_launch_min(vlbm_server* srv, int64_t nodes);
vlbm_status vlbm_server_destroy(vlbm_server* srv);

/* --------------------------------------------------------------- misc --- */
const char* vlbm_last_error(void);     /* thread-local message of the last failure */
int vlbm_abi_version(void);
/* Autotuner (no counterpart in the reference, whose launch shape is fixed at
 * compile time, var.h:124): times the fused step on a copy of the state for
 * each launch shape (64 / 128 / 256 threads per block: the variant returned)
 * and, when the configuration leaves the layout to the library
 * (VLBM_LAYOUT_AUTO) and NZ is even, for each tile a thread advances (one
 * node in the natural layout, the node pair (z, z + NZ/2) in the z-paired one);
 * the state is restored, in the fastest layout, and the fastest shape is
 * kept.  vlbm_info.layout reports the layout in use; checkpoints record it, so
 * an image saved before an autotune that changed the layout loads only into
 * a simulation in the same layout. */
vlbm_status vlbm_autotune(vlbm_sim* sim, int32_t* chosen_variant);
/* Move the state into another population layout (VLBM_LAYOUT_NATURAL, or
 * VLBM_LAYOUT_ZPAIR for an even NZ, in blocks of 32 pair-nodes where NX is a
 * multiple of 32): the stored values are copied, so the state is unchanged,
 * and the layout is kept by later autotuning.  No counterpart in the reference,
 * which has one layout (idxPop, globalFunctions.h:111-147).  Allocates a
 * temporary copy of the population array. */
vlbm_status vlbm_set_layout(vlbm_sim* sim, int32_t layout);
/* Force a kernel launch variant (0 = autotuned default). */
vlbm_status vlbm_set_variant(vlbm_sim* sim, int32_t variant);

/* ------------------------------------------------------ z-slab halos --- */
/* One lattice split along z over several GPUs, one slab (and one process) per
 * GPU; replaces the N_GPUS slabs with a ghost plane and the per-step
 * population transfer between neighbouring GPUs (gpuPopulationsTransfer,
 * lbm.cu:601-657, called from main.cu:336-350).  A slab of n planes is a
 * simulation of n + 2 planes whose planes 0 and n + 1 are ghost copies of the
 * neighbouring slabs' edge planes, marked unused in the node map
 * (vlbm_build_node_map_planes).  The in-place step touches other nodes only in
 * its odd phase (vlbm_info.aa_parity == 1), so slabs exchange only around odd
 * steps: before it, plane 1's c_z = +1 and plane n's c_z = -1 populations go
 * to the neighbours' ghost planes n + 1 and 0; after it, the ghost planes'
 * c_z = -1 and c_z = +1 populations go back to the neighbours' planes n and 1.
 * A message is the stored values of the populations with c_z == dz (dz = +1 or
 * -1) of one plane, [k][ny][nx] with k over those populations in lattice order
 * (5 for D3Q19, 9 for D3Q27), in the storage type; the same bytes whatever
 * the layout.  Pack and unpack are asynchronous on the simulation's stream;
 * dst / src are device pointers of vlbm_halo_bytes bytes. */
vlbm_status vlbm_halo_bytes(vlbm_sim* sim, size_t* bytes);
vlbm_status vlbm_halo_pack(vlbm_sim* sim, int32_t z, int32_t dz, void* dst);
vlbm_status vlbm_halo_unpack(vlbm_sim* sim, int32_t z, int32_t dz, const void* src);
/* The same for a slab's two messages of one exchange in one launch. */
vlbm_status vlbm_halo_pack2(vlbm_sim* sim, int32_t z0, int32_t dz0, void* dst0, int32_t z1, int32_t dz1,
                            void* dst1);
vlbm_status vlbm_halo_unpack2(vlbm_sim* sim, int32_t z0, int32_t dz0, const void* src0, int32_t z1, int32_t dz1,
                              const void* src1);
/* The builder's words for planes z_first .. z_first + n_planes - 1 of an
 * nx x ny x nz lattice, taken modulo nz (so z_first = z0 - 1 and n_planes =
 * n + 2 give a slab with its ghost planes); n must be nx*ny*n_planes.  The
 * caller marks the ghost planes unused (word 0) before vlbm_set_node_map. */
vlbm_status vlbm_build_node_map_planes(int builder, int nx, int ny, int nz, int z_first, int n_planes,
                                       uint32_t* map_out, size_t n);

#ifdef __cplusplus
}
#endif
#endif /* VLBM_H */
