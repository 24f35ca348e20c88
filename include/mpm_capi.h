/*
 * mpm_capi.h -- C ABI of the B200 MPM workpiece step (libmpm_b200.so).
 *
 * Plain C types only: pointers, sizes, scalars.  Every function returns an
 * mpm_status; a failed call leaves a message for mpm_last_error().  Nothing
 * calls exit() or traps the GPU.  A handle is driven by one host thread at a
 * time; device work goes on the stream given to mpm_create (or the handle's
 * own stream) and is asynchronous except where a function says it
 * synchronises.
 *
 * Each entry point names the reference interface it replaces.  The reference
 * solver is class edgepredict::MPMSolver (include/MPMSolver.cuh:76-268) behind
 * IPhysicsSolver / IMetricsProvider / IThermalCoupling
 * (include/IPhysicsSolver.h:24-149).
 */
#ifndef MPM_CAPI_H
#define MPM_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPM_ABI_VERSION 1

typedef enum mpm_status {
    MPM_OK = 0,
    MPM_INVALID_ARG = 1,
    MPM_OOM = 2,
    MPM_CUDA_ERROR = 3,
    MPM_NUMERIC = 4,      /* NaN/Inf in the state, or a Newton return that did not converge */
    MPM_OUT_OF_GRID = 5,
    MPM_TIMEOUT = 6,      /* a bounded device-side wait gave up */
    MPM_NOT_SUPPORTED = 7,
    MPM_CAPACITY = 8,     /* more particles or instances than the handle holds */
    MPM_CANCELLED = 9     /* a served request cancelled by mpm_server_cancel */
} mpm_status;

/* Particle status codes: ParticleStatus, include/Types.h:37-43. */
enum { MPM_ACTIVE = 0, MPM_INACTIVE = 1, MPM_CHIP = 2, MPM_BOUNDARY = 3, MPM_FIXED = 4 };

enum { MPM_PREC_F32 = 0, MPM_PREC_F64 = 1 };
enum { MPM_TOOL_NONE = 0, MPM_TOOL_RASTER = 1, MPM_TOOL_SDF_STICKY = 2, MPM_TOOL_SDF_SLIP = 3 };
enum { MPM_SHAPE_CYLINDER_Y = 0, MPM_SHAPE_WEDGE_Y = 1 };
enum { MPM_PLAST_EXPLICIT = 0, MPM_PLAST_NEWTON = 1 };
enum { MPM_SCHED_SPLIT = 0, MPM_SCHED_FUSED = 1 };

/*
 * Per-instance parameters.  Replaces MPMKernelConfig (include/MPMSolver.cuh:29-74)
 * plus the solver fields MPMSolver::initialize fills (src/MPMSolver.cu:832-915),
 * with the grid given explicitly instead of the hard-wired 0.2 m cube.
 * Temperatures may be in K or degC: only (T - Tamb)/(Tm - Tamb) and
 * differences enter the physics.
 */
typedef struct mpm_params {
    int32_t abi_version;       /* MPM_ABI_VERSION */
    int32_t precision;         /* MPM_PREC_F32 (bulk FP32) or MPM_PREC_F64 */
    /* grid: node (i,j,k) at origin + (i,j,k)*dx, i < nx ... (each >= 8) */
    int32_t nx, ny, nz;
    int32_t plasticity;        /* MPM_PLAST_EXPLICIT (reference return) or MPM_PLAST_NEWTON */
    double dx;
    double origin[3];
    /* particles: uniform mass and initial volume per instance */
    double particle_mass, particle_volume;
    /* elasticity and heat */
    double E, nu, rho_phys, cp, beta, Tm, Tamb;
    /* Johnson-Cook flow stress, reference strain rate, kinematic hardening */
    double jc_A, jc_B, jc_n, jc_C, jc_m, edot0, H_kin;
    /* Johnson-Cook damage */
    double D1, D2, D3, D4, D5, D_th;
    /* grid boundary: fixture layer (applyFixtureBCKernel), gravity, empty-node mass */
    double fixture_thickness, fixture_damping, gravity_z, mass_threshold;
    /* APIC: C = apic_dinv_factor/dx^2 * B, then C *= apic_decay (reference: 3, 0.99) */
    double apic_dinv_factor, apic_decay;
    /* explicit-return caps (reference: 0.05, 50 K) */
    double deps_cap, dT_cap;
    /* level of detail (lodClassifyKernel); radii about the tool tip */
    int32_t lod_enabled;
    int32_t chip_every;        /* chip separation every n-th step (reference: 2); 0 disables */
    double lod_active_r, lod_near_r;
    double newton_tol;         /* relative residual of the Newton return */
    int32_t newton_maxit;
    int32_t schedule;          /* MPM_SCHED_FUSED (default) or MPM_SCHED_SPLIT */
    int32_t sort_every;        /* re-bin particles every n steps (0: default) */
    int32_t threads_per_block; /* CTA size of the step kernel (0: default 128) */
    /* Particle-side tool contact, restating xpbdContactSDFKernel
     * (src/ContactSolver.cu:797-923) on the analytic tool SDF, after the move
     * of every contact_every-th step (0: off): particles within contact_radius
     * of the tool surface are pushed out to it, lose an approaching normal
     * velocity, take Coulomb friction and are heated by (1 - heat partition)
     * of the friction work.  Reference defaults (ContactConfig,
     * include/ContactSolver.cuh:30-34): 0.2 mm, 0.3, 0.5. */
    int32_t contact_every;
    int32_t _pad_contact;
    double contact_radius, contact_friction, contact_heat_partition;
    /* Adiabatic shear band heating, restating AdiabaticShearModel::update
     * (src/AdiabaticShearModel.cu:262-279: applyAdiabaticHeatingKernel,
     * :104-177), after the move of every step and before chip separation, as
     * MPMSolver::step runs it (src/MPMSolver.cu:1130-1132); asb_enabled = 0:
     * off (the reference never enables it).  An ACTIVE particle heated more
     * than asb_touch_rise above Tamb whose strain rate reaches
     * max(asb_critical_rate / 2, 5000 /s) is heated by
     * asb_taylor_quinney * sigma_vM * edot * dt / (rho_phys * cp) (at most
     * 100 K), with T capped at asb_max_temp_ratio * Tm; a per-particle counter
     * of consecutive such steps (0..10) drives the reference's localisation
     * factor.  Reference defaults (AdiabaticShearConfig, include/Types.h:90-94):
     * 1e4 /s, 0.9, 0.9; the reference's guard T <= 25.5 degC with its 25 degC
     * ambient is a rise of 0.5. */
    int32_t asb_enabled;
    int32_t _pad_asb;
    double asb_critical_rate, asb_taylor_quinney, asb_max_temp_ratio, asb_touch_rise;
    /* Grid heat conduction as MPMWorkpieceSolver does it, on this solver's
     * quadratic weights (heat_conduction = 0: off; MPMSolver conducts no
     * heat).  P2G scatters T m with the mass (src/MPMWorkpieceSolver.cu:118);
     * between P2G and G2P every node with m >= 1e-15 takes one explicit step
     * T += alpha dt lap(T) / dx^2 of T = (T m)/m, alpha = thermal_conductivity
     * / (rho_phys cp), 7-point Laplacian, no flux through the domain faces, an
     * empty neighbour counted as T = 0, T >= 0 (mpmDiffuseTemperatureKernel,
     * :208-262); G2P then sets the temperature of every particle that is not
     * FIXED to the weight-normalised mean over the nodes with m > 1e-18,
     * clamped to [Tamb, Tm] (:282-306).  Temperatures are absolute here (the
     * empty-node T = 0 is the unit's zero).  Reference default
     * (MPMMaterialParams::thermalConductivity,
     * include/MPMWorkpieceSolver.cuh:88): 42.6 W/(m K). */
    int32_t heat_conduction;
    int32_t _pad_heat;
    double thermal_conductivity;
} mpm_params;

/* Fill p with the reference defaults (MPMKernelConfig / Config.h defaults,
 * reference-compatible kinematics).  Grid and particle fields are zeroed. */
mpm_status mpm_params_default(mpm_params *p);

/*
 * Rigid tool.  The reference rasterises FEM tool nodes onto the grid
 * (MPMSolver::setToolNodes, include/MPMSolver.cuh:86-89; rasterizeToolKernel
 * src/MPMSolver.cu:444-473; applyGridCollisionKernel :475-492).  Here the tool
 * is a rigid body with reference point p(t) = position + velocity*(t - t_set):
 *   MPM_TOOL_RASTER     sample offsets from the reference point, rasterised
 *                       exactly as the reference does (parity mode);
 *   MPM_TOOL_SDF_STICKY analytic SDF; nodes with phi <= 0 take the tool velocity;
 *   MPM_TOOL_SDF_SLIP   analytic SDF; approaching normal relative velocity removed.
 * tip_dz: z of the tool tip relative to the reference point (chip separation
 * and LOD use the tip, as MPMSolver::setToolPosition does).
 */
typedef struct mpm_tool_desc {
    int32_t mode;
    int32_t shape;
    double position[3];
    double velocity[3];
    double radius;             /* cylinder radius, or wedge edge radius */
    double rake, clearance;    /* wedge angles (rad) */
    double tip_dz;
    int32_t n_samples;         /* MPM_TOOL_RASTER: sample offsets (host arrays) */
    int32_t _pad;
    const double *sample_dx, *sample_dy, *sample_dz;
} mpm_tool_desc;

/*
 * Host particle arrays in the reference's units (m, m/s, Pa, degC/K).
 * Matrices row-major [n][9] (F, F_p, C as MPMParticle, include/Types.h:219-225),
 * symmetric tensors [n][6] as xx,yy,zz,xy,xz,yz.  `elem` = 8 (double) or 4 (float)
 * for every floating field.  A NULL field reads as its MPMParticle default on
 * upload and is skipped on download.
 */
typedef struct mpm_particles_soa {
    int32_t elem;
    int32_t _pad;
    void *x, *y, *z, *vx, *vy, *vz;
    void *F, *Fp, *C, *stress, *backstress;
    void *plastic_strain, *strain_rate, *temperature, *damage, *residual_stress;
    int32_t *status, *id;
} mpm_particles_soa;

typedef struct mpm_metrics {
    /* reference-compatible (computeParticleStatsKernel, src/MPMSolver.cu:729-788) */
    double ref_max_stress, ref_max_temperature, ref_kinetic, ref_internal;
    /* conservation, FP64 reductions over particles that are not INACTIVE */
    double mass, momentum[3], kinetic, internal_elastic, thermal;
    double max_temperature, max_von_mises, max_plastic_strain, mean_plastic_strain;
    int64_t n_active, n_chip, n_fixed, n_inactive;
    double bounds_min[3], bounds_max[3];   /* ACTIVE and CHIP particles */
    /* counters of the whole handle (all instances of a batch), cumulative */
    int64_t n_escaped;                     /* particle updates done off their bin tile */
    int64_t n_sorts;                       /* re-bins so far */
    int64_t n_yielded;                     /* particle updates that took a plastic return */
    int64_t n_contacts;                    /* particle contact corrections */
    double contact_work, contact_force;    /* friction work (J) and normal force (N) summed over them */
    int64_t n_asb_heated;                  /* particle updates heated by the adiabatic shear model */
} mpm_metrics;

typedef struct mpm_handle mpm_handle;

/* Replaces MPMSolver::MPMSolver + initialize(Config) (src/MPMSolver.cu:832-915):
 * validates p, allocates device state for up to `capacity` particles.
 * stream: a cudaStream_t or NULL for a handle-owned stream. */
mpm_status mpm_create(const mpm_params *p, int64_t capacity, void *stream, mpm_handle **out);
/* Replaces MPMSolver::~MPMSolver / freeMemory (src/MPMSolver.cu:933-964). */
mpm_status mpm_destroy(mpm_handle *h);

/* Replaces MPMSolver::initializeParticleBox (src/MPMSolver.cu:1297-1336) with a
 * seeded, jittered box: cells [c0, c1) (cell units from the grid origin),
 * ppc particles per cell, candidate k of a cell at a Philox4x32-10 uniform
 * point (keyed by seed, instance, cell, k) of its own stratum of the cell --
 * for ppc <= 8 one octant per candidate in a fixed order, for larger ppc one
 * sub-cell of the n^3 grid (n even) -- so that, as on the reference's regular
 * lattice, every interior stencil-base cell holds exactly ppc particles;
 * cells whose lowest `fixed_layers` z-layers are FIXED_BOUNDARY; particles
 * inside the tool at t=0 are not kept.  Generated on the device. */
mpm_status mpm_init_box(mpm_handle *h, const int32_t c0[3], const int32_t c1[3], int32_t ppc, uint64_t seed,
                        uint32_t instance, int32_t fixed_layers, double T0, const mpm_tool_desc *tool_at_t0);

/* Upload n particles from host arrays (replaces copyToDevice via
 * getHostParticles/updateParticlesFromHost, include/MPMSolver.cuh:185-186). */
mpm_status mpm_upload(mpm_handle *h, const mpm_particles_soa *host, int64_t n);
/* Download the particles in upload order (replaces getParticles,
 * src/MPMSolver.cu:1383-1386).  Synchronises. */
mpm_status mpm_download(mpm_handle *h, mpm_particles_soa *host);
/* Copy the particles, in upload order, into an array of the reference's
 * MPMParticle layout (include/Types.h:199-266, 504 bytes) for ContactSolver,
 * CFD and the exporters.  dst is host or device memory. Synchronises. */
mpm_status mpm_export_aos(mpm_handle *h, void *dst, int64_t dst_bytes);

/* Fields of an MPMParticle array that mpm_import_aos reads back. */
enum {
    MPM_AOS_POSITION = 1,     /* x, y, z */
    MPM_AOS_VELOCITY = 2,     /* vx, vy, vz */
    MPM_AOS_TEMPERATURE = 4,  /* temperature */
    MPM_AOS_STATUS = 8,       /* status (0..4; a record outside that range keeps its status) */
    MPM_AOS_EXT_FORCE = 16,   /* ext_fx, ext_fy, ext_fz: a body force for the next step only */
    MPM_AOS_WRITABLE = 31     /* all of the above */
};

/* The way back from mpm_export_aos.  The reference's consumers of the
 * particle array write the solver's own d_particles in place:
 * ContactSolver::resolveContacts (xpbdContactSDFKernel, src/ContactSolver.cu:
 * 797-923, launched at :1130-1147) moves positions, velocities and
 * temperatures; CFD chip coupling adds drag to ext_f and cooling to the
 * temperature (src/CFDSolverGPU.cu:1347-1400, registered at
 * src/SimulationEngine.cpp:1008-1013).  This reads the `fields` of an array
 * of n records (n = the workpiece's particles, in upload order, as
 * mpm_export_aos wrote it; src is host or device memory of at least
 * n * 504 bytes) back into the workpiece:
 *   - a position, velocity or temperature equal to what mpm_export_aos would
 *     write now is left as it is (an unmodified array imports as a no-op, bit
 *     for bit); moved particles are re-binned before the next step;
 *   - the external force acts in the next step's P2G on every particle that
 *     is not INACTIVE, as the reference's p2gKernel adds w * ext_f to the
 *     node force (src/MPMSolver.cu:410-417), and is then cleared
 *     (resetExternalForceKernel, :682-688).
 * Synchronises; MPM_INVALID_ARG when a record's status is outside 0..4
 * (those records keep their status, the other fields are imported). */
mpm_status mpm_import_aos(mpm_handle *h, const void *src, int64_t src_bytes, uint32_t fields);

/* Replaces setToolNodes / setToolPosition (include/MPMSolver.cuh:86-89, :171). */
mpm_status mpm_set_tool(mpm_handle *h, const mpm_tool_desc *tool);

/* The raster tool read straight from the FEM tool's node records in device
 * memory (the reference's FEMNodeGPU, include/Types.h:316-379, or any record
 * with double x, y, z and vx, vy, vz fields), as rasterizeToolKernel reads
 * them (src/MPMSolver.cu:444-473), with the sub-step blend of
 * interpolateToolNodesKernel (:494-504) done on the device: no host copy of
 * the nodes and no synchronisation per step. */
typedef struct mpm_tool_nodes {
    const void *start;    /* device records at the start of the blended motion, or NULL (no blend) */
    const void *end;      /* device records the step reads (the current FEM nodes) */
    int32_t n;            /* records */
    int32_t stride;       /* bytes from one record to the next (sizeof(FEMNodeGPU)) */
    int32_t off_pos[3];   /* byte offsets of x, y, z (double) in a record */
    int32_t off_vel[3];   /* byte offsets of vx, vy, vz (double) */
    double alpha0;        /* blend weight of the first step after this call */
    double dalpha;        /* added per step */
} mpm_tool_nodes;

/* The grid boundary of raster mode from device node records (mode becomes
 * MPM_TOOL_RASTER; the tool descriptor's pose still drives chip separation
 * and LOD).  At the j-th step after the call (counted across step calls),
 * node q sits at end_q when start is NULL, else at start_q + a (end_q -
 * start_q) with a = alpha0 + j * dalpha; it marks the 2x2x2 grid nodes from
 * round((x - origin) / dx), and a marked grid node takes the velocity of the
 * highest-indexed tool node that marks it (the reference's last writer is
 * whichever thread ran last).  The velocity is end_q's: the reference reads
 * it from its blend buffer, whose velocity fields interpolateToolNodesKernel
 * never writes (:494-504).  Both arrays must stay valid and unchanged while
 * the steps that read them run.  nodes = NULL returns to the descriptor's
 * sample offsets. */
mpm_status mpm_set_tool_nodes(mpm_handle *h, const mpm_tool_nodes *nodes);

/*
 * Voxel signed-distance field of the tool for the particle-side contact
 * (mpm_params.contact_every > 0).  Replaces ToolSDF::build / createTexture
 * (src/ToolSDF.cu:212-280, :534-567) and setToolTransform (:569-576): the
 * values are the tool's signed distances (m, negative inside) at the voxel
 * centres origin + (i + 1/2) voxel of the tool frame, whose origin follows the
 * tool's reference point and which is rotated by `angle` about z.  The step
 * then resolves contact as xpbdContactSDFKernel (src/ContactSolver.cu:797-923)
 * does, sampling the field through a trilinear 3D texture like the
 * reference's; without one it uses the analytic tool SDF.  values are copied
 * (host memory, x fastest); NULL sdf removes the field.
 */
typedef struct mpm_tool_sdf {
    int32_t nx, ny, nz;        /* voxels per axis, 2 .. 1024 */
    int32_t _pad;
    const float *values;
    float origin[3];           /* corner of voxel (0,0,0) in the tool frame (m) */
    float voxel;               /* voxel edge (m) */
    float angle;               /* rotation of the tool frame about z (rad) */
    float _pad2;
} mpm_tool_sdf;

mpm_status mpm_set_tool_sdf(mpm_handle *h, const mpm_tool_sdf *sdf);

/*
 * The voxel SDF of a closed tool mesh, built as ToolSDF does
 * (src/ToolSDF.cu:212-280 build, :348-377 buildFromVerts, :379-532
 * computeSDFCPU): the mesh bounding box grown by `padding` (m), an isotropic
 * voxel of the longest extent / voxels_per_axis, extent / voxel + 2 voxels
 * per axis (at most 256); each triangle's distance to the voxel centres of its
 * box grown by one voxel below and two above, the sign within two voxels of
 * the surface from the nearest triangle's normal, three passes that reach the
 * voxels no box covered (nearest |distance| + half a voxel) and a large
 * distance beyond.  Distances and signs are computed on the current GPU, the
 * passes on the host.  verts [n_verts][3], tris [n_tris][3], normals
 * [n_tris][3] or NULL ((b - a) x (c - a) normalised).  With values NULL only
 * desc is filled (nx, ny, nz, origin, voxel; angle 0); with values of
 * nx*ny*nz floats the field is written there and desc->values points to it.
 */
mpm_status mpm_tool_sdf_build(const float *verts, int32_t n_verts, const int32_t *tris, int32_t n_tris,
                              const float *normals, double padding, int32_t voxels_per_axis, mpm_tool_sdf *desc,
                              float *values);

/* Replaces MPMSolver::step (src/MPMSolver.cu:1062-1168): nsteps steps of dt.
 * Asynchronous on the handle's stream. */
mpm_status mpm_step(mpm_handle *h, double dt, int32_t nsteps);

/* The constants of the reference's other MPM solver, MPMWorkpieceSolver
 * (MPMMaterialParams, include/MPMWorkpieceSolver.cuh:60-83), that mpm_params
 * does not carry. */
typedef struct mpm_workpiece_params {
    double failure_strain;           /* damage += rate dt / max(failure_strain, 1e-3) */
    double critical_plastic_strain;  /* ACTIVE -> CHIP at this plastic strain */
    double thermal_chip_ratio;       /* ACTIVE -> CHIP at T >= ratio * Tm */
    double tool_contact_radius;      /* a grid node within this of a tool sample is in contact */
    double contact_damping;          /* contact heating 0.5 m vn^2 * damping */
    double max_contact_temp_rise;    /* per-step cap of contact and plastic heating */
    int32_t thermal_clamp;           /* the cap on (1) or off (0) */
    int32_t _pad;
} mpm_workpiece_params;

/* Switches the handle's step to MPMWorkpieceSolver::step
 * (src/MPMWorkpieceSolver.cu:727-781), the reference's other MPM solver,
 * which its engine never constructs: trilinear PIC transfers (:52-134,
 * :264-306), the grid update with the fixture and the nearest-tool-sample
 * normal projection and contact heating (:136-192), the grid diffusion step
 * when thermal_conductivity > 0 (:208-262), a hypoelastic stress rate with
 * the Johnson-Cook radial return at the old plastic strain, kinematic
 * hardening, strain-rate damage and the CHIP criteria (:308-395), and its
 * chip separation on even steps (:667-725).  mpm_params supplies the grid,
 * E and nu, rho_phys (its density), cp, Tm, Tamb (its reference
 * temperature), the Johnson-Cook constants, edot0, D_th, H_kin, the fixture
 * thickness and the conductivity; the tool samples of an MPM_TOOL_RASTER
 * descriptor are its tool samples, at the tool's pose each step; the tool tip
 * for the chip separation is pose z + tip_dz.  mpm_apply_external_force
 * takes its form (the whole force on ACTIVE particles within the radius,
 * :402-413).  The grid stays the handle's (the solver's rebuild of its grid
 * from the particle bounds is host-side domain management).  NULL returns to
 * MPMSolver's semantics.  Its kernels sum with atomics as the reference's
 * do (FP64 runs agree to 1e-15, FP32 to summation order) whatever the
 * launch config's deterministic flag says.  Not for a batch of more than one
 * workpiece. */
mpm_status mpm_set_workpiece_semantics(mpm_handle *h, const mpm_workpiece_params *params);

/* Replaces getStableTimeStep (src/MPMSolver.cu:1170-1178): cfl*dx/sqrt(E/rho). */
mpm_status mpm_stable_dt(const mpm_handle *h, double cfl, double *dt);

/* Replaces syncMetrics + getters (src/MPMSolver.cu:1239-1259,
 * include/MPMSolver.cuh:135-139) and getBounds (:1232-1237).  Synchronises;
 * also reports a device-side error (MPM_NUMERIC / MPM_TIMEOUT). */
mpm_status mpm_sync_metrics(mpm_handle *h, mpm_metrics *out);

/* No counterpart in the reference (which copies every particle to the host to
 * compute these, src/MPMSolver.cu:1239-1259).  The metrics of mpm_sync_metrics
 * for n particles held in DEVICE memory in the reference's MPMParticle layout
 * (include/Types.h:199-266, 504 bytes each: the reference's own d_particles,
 * or mpm_export_aos written to device memory), with no handle and no
 * allocation, for callers that cannot allocate device memory.  Mass, volume,
 * density and temperature are read per record; p supplies E, nu, cp and Tamb.
 * n_escaped, n_sorts and n_yielded are 0.
 *   - Scratch is a 1 MiB static device array inside the library; n above
 *     67,108,864 is refused with MPM_CAPACITY.  Nothing has to be zeroed first.
 *   - Every call looks up the scratch's address in the current context of
 *     the current device (the first call there also loads the library's
 *     kernels), so a device reset or another current context is followed.
 *     The call synchronises its stream: make it outside stream capture.
 *   - Calls on one device must not overlap (two host threads, or two streams
 *     in flight at once): they share the scratch and race.
 *   - stream: a cudaStream_t or NULL (legacy default stream).  Synchronises
 *     that stream before returning. */
mpm_status mpm_metrics_aos_noalloc(const mpm_params *p, const void *d_particles, int64_t n, void *stream,
                                   mpm_metrics *out);

/* Replaces setDynamicMassScaling (src/MPMSolver.cu:1211-1225): particle mass
 * becomes rho_phys*factor*volume (never below rho_phys*volume). */
mpm_status mpm_set_mass_scaling(mpm_handle *h, double factor);

/* Replaces applyExternalForce (src/MPMSolver.cu:1422-1431): a force with
 * linear falloff inside a sphere, applied during the next step only. */
mpm_status mpm_apply_external_force(mpm_handle *h, const double center[3], double radius, const double force[3]);

/* Replaces setParticleTemperatures (src/MPMSolver.cu:1267-1277): count <= n
 * temperatures in upload order. */
mpm_status mpm_set_temperatures(mpm_handle *h, const double *temperatures, int64_t count);

mpm_status mpm_get_counts(const mpm_handle *h, int64_t *n_particles, int64_t *n_steps, double *time);
mpm_status mpm_get_stream(const mpm_handle *h, void **stream);
/* Replaces reset() (src/MPMSolver.cu:1227-1230): time and step counter to 0. */
mpm_status mpm_reset_clock(mpm_handle *h);

/*
 * Batched form.  No counterpart in the reference, which runs one MPMSolver
 * per simulation (src/main.cpp:307).  One handle holds many independent
 * workpieces (instances), each with its own grid, material, tool and time
 * step; every step of all of them is one persistent launch over the bins of
 * all instances.  The single-instance functions above act on instance 0 of
 * a batch handle (mpm_step: the same dt for every instance).
 */
mpm_status mpm_batch_create(const mpm_params *params, const int64_t *capacities, int32_t n_instances, void *stream,
                            mpm_handle **out);
mpm_status mpm_batch_count(const mpm_handle *h, int32_t *n_instances);
mpm_status mpm_batch_init_box(mpm_handle *h, int32_t inst, const int32_t c0[3], const int32_t c1[3], int32_t ppc,
                              uint64_t seed, uint32_t instance_key, int32_t fixed_layers, double T0,
                              const mpm_tool_desc *tool_at_t0);
mpm_status mpm_batch_upload(mpm_handle *h, int32_t inst, const mpm_particles_soa *host, int64_t n);
mpm_status mpm_batch_download(mpm_handle *h, int32_t inst, mpm_particles_soa *host);
mpm_status mpm_batch_export_aos(mpm_handle *h, int32_t inst, void *dst, int64_t dst_bytes);
mpm_status mpm_batch_import_aos(mpm_handle *h, int32_t inst, const void *src, int64_t src_bytes, uint32_t fields);
mpm_status mpm_batch_set_tool(mpm_handle *h, int32_t inst, const mpm_tool_desc *tool);
mpm_status mpm_batch_set_tool_sdf(mpm_handle *h, int32_t inst, const mpm_tool_sdf *sdf);
mpm_status mpm_batch_set_tool_nodes(mpm_handle *h, int32_t inst, const mpm_tool_nodes *nodes);
/* nsteps steps of every instance; dt[i] is instance i's step (n_instances values). */
mpm_status mpm_batch_step(mpm_handle *h, const double *dt, int32_t nsteps);
mpm_status mpm_batch_sync_metrics(mpm_handle *h, int32_t inst, mpm_metrics *out);
/* Failure detection per workpiece (the reference has one host-side health
 * check per simulation, SimulationHealthMonitor::check, which halts it:
 * include/SimulationHealthMonitor.h:321-328).  Every instance has an error
 * word that only its own failures mark: in the step kernel, a particle whose
 * position is not finite (the kill zone deactivates it, as the reference's
 * does) or a Newton return that did not converge; a NaN or Inf velocity or
 * stress reaches the positions through the grid within one step.
 * mpm_batch_sync_metrics also marks the word when a sum over the live
 * particles (mass, momentum, energies, plastic strain) is not finite.
 * status[i] (n >= the instance count) receives MPM_OK or MPM_NUMERIC per
 * instance (MPM_TIMEOUT for all when a bounded device wait gave up).
 * mpm_batch_sync_metrics, mpm_batch_download and mpm_export_aos report the
 * status of their own instance (the data is written all the same), so a
 * failed workpiece can be dropped (mpm_batch_change) while the others run
 * on.  mpm_batch_upload and mpm_batch_init_box clear the instance's word;
 * the word moves with its instance across mpm_batch_change.  Works on a
 * plain handle too (one instance).  Synchronises the handle's stream. */
mpm_status mpm_batch_instance_status(mpm_handle *h, int32_t *status, int32_t n);

/* Checkpoint and resume of one workpiece (no counterpart in the reference,
 * which serialises no state).  A checkpoint is a versioned header (format
 * version, ABI version, precision, step count, clock, mpm_params, tool) and
 * the instance's particle state exactly as it is held on the device, with a
 * 64-bit checksum; a serving loop can preempt a workpiece and resume it later,
 * in this handle or another.  Loading needs an instance of the same
 * precision and grid size (nx, ny, nz) with room for the particles; it
 * replaces the instance's parameters, tool, clock and particles, and clears
 * its error word.  A voxel tool SDF (mpm_set_tool_sdf) is not part of the
 * checkpoint: set it again after loading.  The state is written to and read
 * from caller memory (host or pinned); _bytes gives the size.  The saved
 * state includes the particles' layout (each one's re-bin key) and the
 * instance's re-bin phase, so the reloaded instance keeps its layout and
 * re-bins at the same steps: a resumed run continues the saving run's sums in
 * the same order.  With the deterministic mode it gives the same bits; with
 * the default atomics it agrees to summation order (FP64 1e-9), as a batch
 * does with its instances run alone.  Single-instance handles use inst 0. */
mpm_status mpm_checkpoint_bytes(mpm_handle *h, int32_t inst, int64_t *bytes);
mpm_status mpm_checkpoint_save(mpm_handle *h, int32_t inst, void *buf, int64_t bytes);
mpm_status mpm_checkpoint_load(mpm_handle *h, int32_t inst, const void *buf, int64_t bytes);
mpm_status mpm_batch_get_counts(const mpm_handle *h, int32_t inst, int64_t *n_particles, int64_t *n_steps,
                                double *time);
/* Drops the n_remove listed instances (their state is freed; the indices of
 * the instances after them shift down) and appends n_add new, empty ones
 * (fill them with mpm_batch_init_box / mpm_batch_upload).  The other
 * instances keep their state and clock.  *first_added (may be NULL) receives
 * the index of the first new instance. */
mpm_status mpm_batch_change(mpm_handle *h, const mpm_params *add, const int64_t *add_capacities, int32_t n_add,
                            const int32_t *remove, int32_t n_remove, int32_t *first_added);

/* Launch shape of the step kernel.  Not part of the physics: any setting
 * gives the same results up to FP32 summation order. */
typedef struct mpm_launch_config {
    int32_t ctas_per_sm;   /* persistent CTAs per SM of the step kernel, 1..8 (default 4) */
    int32_t sort_every;    /* re-bin every n steps, 1..1024 (default mpm_params.sort_every) */
    int32_t use_graph;     /* replay each step call's launches from a captured CUDA graph */
    /* 1 (the default): deterministic mode (no counterpart in the reference,
     * whose P2G sums with FP64 atomics in arrival order).  The results are
     * the same bit for bit on every run, every launch shape and every split
     * of the steps into calls, alone or in a batch.  0: each work item adds
     * its node tile to the grid with FP32 atomics (about 1 % faster; the
     * last bits vary from run to run).  The deterministic mode runs the same
     * fused step kernel with three changes: each work item stores its node tile
     * and one thread per grid node adds the stored tiles of the bins that
     * cover it in a fixed order (no float atomics; one extra launch per step);
     * a particle whose stencil left its bin's tile adds to the grid in 2^-40
     * particle-mass fixed point with integer atomics; and the re-bin's order
     * within each cell (which it uses in both modes) is the order of the old
     * slots.  Holds 5 x 216 reals per bin and 5 x 8 bytes per grid node more;
     * every option runs in it (graphs included) except the
     * MPMWorkpieceSolver semantics (MPM_NOT_SUPPORTED at the step). */
    int32_t deterministic;
    /* FP32 particles staged per pass of the step kernel: 128, 256 or 512
     * (0: the default, 128).  A larger pass halves the passes' barriers and
     * node-tile adds and takes more shared memory per CTA (512: three CTAs
     * per SM).  FP64 and the kernel variant with the adiabatic shear model,
     * heat conduction or the voxel contact stage 128 whatever this says. */
    int32_t pass_size;
} mpm_launch_config;
mpm_status mpm_get_launch_config(const mpm_handle *h, mpm_launch_config *out);
mpm_status mpm_set_launch_config(mpm_handle *h, const mpm_launch_config *cfg);
/* Picks the launch shape by timing real steps (dt[i] per instance, counted
 * like any other steps): first the pass size (128, 256, 512 FP32 particles,
 * 16 steps each at the current CTAs and cadence), then, at the fastest pass
 * size, every CTAs per SM in {2,3,4} x re-bin every {8,16,32} steps over one
 * re-bin period each (216 steps in all).  Keeps the fastest; *chosen (may be
 * NULL) receives it. */
mpm_status mpm_autotune(mpm_handle *h, const double *dt, mpm_launch_config *chosen);

/*
 * Serving loop (continuous batching).  No counterpart in the reference.
 * Solve requests -- a workpiece, its tool and a number of steps -- are
 * submitted at any time; each mpm_server_tick retires finished requests,
 * admits queued ones in arrival order while their footprint fits the device
 * pools reserved from hbm_budget_bytes (88 % particle state, 8 % grids, 3 %
 * sort keys, 0.5 % bin tables), and advances every resident request by the
 * same number of steps (at most max_chunk) in one batch step call, so
 * requests admitted while others run share their launches.  The state of
 * every resident request stays on the device.  submit and poll may be
 * called from other threads than tick; tick from one thread at a time.
 */
typedef struct mpm_request {
    mpm_params params;         /* grid, material and options of this workpiece */
    mpm_tool_desc tool;        /* tool at t = 0: MPM_TOOL_NONE or an SDF mode */
    int32_t c0[3], c1[3];      /* workpiece box in cells (as mpm_init_box) */
    int32_t ppc, fixed_layers;
    uint64_t seed;
    uint32_t instance_key;
    int32_t nsteps;
    double dt, T0;
} mpm_request;

enum { MPM_REQ_UNKNOWN = 0, MPM_REQ_QUEUED = 1, MPM_REQ_RUNNING = 2, MPM_REQ_DONE = 3, MPM_REQ_FAILED = 4,
       MPM_REQ_CANCELLED = 5 };

typedef struct mpm_result {
    int32_t state;             /* MPM_REQ_* */
    int32_t status;            /* mpm_status of a FAILED (or CANCELLED) request */
    int64_t n_particles;
    int64_t steps_done;
    double t_submit, t_admit, t_done;   /* seconds on the server's clock */
    mpm_metrics metrics;       /* at completion (DONE) */
} mpm_result;

typedef struct mpm_server_config {
    int32_t precision;         /* MPM_PREC_F32 or MPM_PREC_F64, for every request */
    int32_t max_chunk;         /* steps per tick at most (0: 50) */
    int64_t hbm_budget_bytes;  /* device memory reserved at creation for resident requests */
    int32_t max_resident;      /* requests resident at once at most (0: 4096) */
    int32_t use_graph;         /* replay the tick's step calls from captured CUDA graphs */
    int32_t backstress;        /* also reserve backstress state (requests with H_kin > 0) */
    int32_t deterministic;     /* 1: step in deterministic mode (mpm_launch_config.deterministic), so a
                                  request's result is the same bit for bit alone and in any mix; the
                                  mode's per-slot scratch is taken from the budget */
    /* admission also stops at this many resident particles (0: the budget
     * alone); fewer resident particles step faster, so requests finish
     * sooner, at the same throughput once the GPU is full */
    int64_t max_resident_particles;
} mpm_server_config;

typedef struct mpm_server_stats {
    int64_t offered, admitted, completed, failed, queued, resident;
    int64_t particle_updates;  /* particles x steps of all requests so far */
    int64_t resident_particles;
    int64_t ticks;
    double busy_seconds;       /* time spent inside mpm_server_tick */
    int64_t cancelled;
    int64_t preempted;         /* preemptions carried out (a request may count more than once) */
} mpm_server_stats;

typedef struct mpm_server mpm_server;
mpm_status mpm_server_create(const mpm_server_config *cfg, void *stream, mpm_server **out);
mpm_status mpm_server_destroy(mpm_server *s);
/* Queues a request; *id identifies it for mpm_server_poll.  MPM_CAPACITY when
 * its footprint can never fit the pools. */
mpm_status mpm_server_submit(mpm_server *s, const mpm_request *req, int64_t *id);
mpm_status mpm_server_tick(mpm_server *s, int32_t *n_resident);
mpm_status mpm_server_poll(mpm_server *s, int64_t id, mpm_result *out);
/* Cancels a request: a queued one leaves the queue at once, a running one is
 * dropped from the device at the next tick (its steps so far are counted);
 * both end in MPM_REQ_CANCELLED with status MPM_CANCELLED.  A request that
 * already ended keeps its state.  May be called from another thread than
 * tick.  A running request whose workpiece fails (its instance error word is
 * set, see mpm_batch_instance_status) ends in MPM_REQ_FAILED with status
 * MPM_NUMERIC at the tick that stepped it and is dropped at the next one;
 * the other requests run on. */
mpm_status mpm_server_cancel(mpm_server *s, int64_t id);
/* Preempts a running request (no counterpart in the reference): the next
 * tick saves its workpiece to host memory as a checkpoint (see
 * mpm_checkpoint_save), drops it from the device, which frees its share of
 * the pools, and queues the request again at the back.  When it is admitted
 * again the checkpoint is loaded in place of a new workpiece, so it resumes
 * at the step it reached, with the same results as an uninterrupted run to
 * summation order.  MPM_INVALID_ARG for an unknown id or a request that is
 * not running.  May be called from another thread than tick. */
mpm_status mpm_server_preempt(mpm_server *s, int64_t id);
mpm_status mpm_server_stats_get(mpm_server *s, mpm_server_stats *out);
/* Device bytes a request holds while resident (host-only arithmetic). */
mpm_status mpm_server_footprint(const mpm_server_config *cfg, const mpm_request *req, int64_t *bytes);

/* Self-test of the bounded device-side wait that guards the step kernel's
 * tile loads (no counterpart in the reference): a one-thread kernel waits on
 * an mbarrier that nothing completes, gives up after limit_ns (1e6..1e9 ns)
 * and records it.  Returns MPM_TIMEOUT when the wait gave up (the expected
 * outcome; the context stays usable), MPM_CUDA_ERROR otherwise.  Synchronises
 * the stream (NULL: legacy default stream). */
mpm_status mpm_selftest_bounded_wait(int64_t limit_ns, void *stream);

/* Bounds-checked build report (no counterpart in the reference, which has
 * no sanitizer runs).  libmpm_b200_checked.so, built with -DMPMB_CHECKED,
 * checks every index its step kernels derive from data (particle slots of a
 * work item, grid nodes of the tile flush and of the off-tile scatter and
 * gather, heat-conduction nodes, the deterministic mode's node sums and
 * stored tiles) before using it; a failed check is counted, the first one's
 * site (1 particle slot, 2 tile flush, 3 scatter, 4 gather, 5 heat scatter,
 * 6 work item, 7 node of the deterministic node sum, 8 its stored tile) and
 * index are kept, and the access is
 * skipped rather than trapped.  This reads the record after synchronising the
 * device, and clears it when reset != 0.  The default library has no checks
 * and returns MPM_NOT_SUPPORTED with zeros. */
mpm_status mpm_check_report(int64_t *violations, int32_t *site, int64_t *index, int32_t reset);

/* Record CUDA events around every launch of the step kernel (enable != 0),
 * for timing the dominant kernel inside a longer run.  mpm_profile_read
 * synchronises, returns the summed device time (ms) and count of the fused
 * G2P+P2G launches (or of all step launches under the split schedule) since
 * the last read, and clears them. */
mpm_status mpm_profile_enable(mpm_handle *h, int32_t enable);
mpm_status mpm_profile_read(mpm_handle *h, double *kernel_ms, int64_t *kernel_launches);

/* Count of the library's own kernel launches issued by this handle so far. */
mpm_status mpm_launch_count(const mpm_handle *h, int64_t *count);

/* Last error message of the handle (or of the library when h is NULL). */
const char *mpm_last_error(const mpm_handle *h);
const char *mpm_status_string(mpm_status s);

#ifdef __cplusplus
}
#endif
#endif
