/*
 * mpm_oracle.h -- CPU FP64 restatement of the EdgePredict MPM workpiece step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle that the CUDA path is checked
 * against; it is never linked into, loaded by, or called from the product
 * library.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg may use it.
 *
 * It follows the reference's engine-wired solver, src/MPMSolver.cu, kernel by
 * kernel (citations per function in mpm_oracle.c), on plain SoA double
 * arrays.  Beyond the reference it restates three extensions of this build
 * with the same arithmetic that the CUDA path uses: an analytic tool SDF
 * boundary (sticky and slip), a consistent Newton return for Johnson-Cook
 * plasticity, and FP64 conservation metrics.
 *
 * Parity pin: the reference ships no tests or golden vectors.  The oracle is
 * pinned against the reference's own CUDA kernels (built from its sources by
 * oracle/Makefile into oracle/_ref/) through the fixtures in tests/golden/.
 */
#ifndef MPM_ORACLE_H
#define MPM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Particle status codes: include/Types.h:37-43 (ParticleStatus). */
enum { ORC_ACTIVE = 0, ORC_INACTIVE = 1, ORC_CHIP = 2, ORC_BOUNDARY = 3, ORC_FIXED = 4 };

/* Tool boundary modes. */
enum {
    ORC_TOOL_NONE = 0,
    ORC_TOOL_RASTER = 1,      /* reference: rasterizeToolKernel + applyGridCollisionKernel */
    ORC_TOOL_SDF_STICKY = 2,  /* analytic SDF, nodes inside take the tool velocity */
    ORC_TOOL_SDF_SLIP = 3     /* analytic SDF, approaching normal velocity removed */
};
enum { ORC_SHAPE_CYLINDER_Y = 0, ORC_SHAPE_WEDGE_Y = 1 };
enum { ORC_PLAST_EXPLICIT = 0, ORC_PLAST_NEWTON = 1 };

struct orc_sdf_grid;

typedef struct orc_params {
    /* background grid: node (i,j,k) sits at origin + (i,j,k)*dx */
    int32_t nx, ny, nz;
    int32_t _pad0;
    double dx;
    double ox, oy, oz;
    /* elasticity and heat */
    double E, nu;
    double rho_phys, cp, beta, Tm, Tamb;
    /* Johnson-Cook flow stress and kinematic hardening */
    double A, B, n, C, m, edot0, Hkin;
    /* Johnson-Cook damage */
    double D1, D2, D3, D4, D5, Dth;
    /* grid boundary conditions */
    double fixture_thickness, fixture_damping, gravity_z, mass_threshold;
    /* APIC: C = factor/dx^2 * B, then C *= decay */
    double apic_dinv_factor, apic_decay;
    /* level of detail (src/MPMSolver.cu:656-676) */
    int32_t lod_enabled;
    int32_t plasticity_mode;
    double lod_active_r, lod_near_r;
    /* explicit-return safety caps (src/MPMSolver.cu:255, :315) */
    double deps_cap, dT_cap;
    /* chip separation every `chip_every` steps (src/MPMSolver.cu:1160) */
    int32_t chip_sep_enabled, chip_every;
    /* rigid tool: reference point p(t) = p0 + v*t */
    int32_t tool_mode, tool_shape;
    double tool_p0[3];
    double tool_v[3];
    double tool_r;          /* cylinder radius, or wedge edge radius */
    double tool_rake;       /* wedge rake angle (rad) */
    double tool_clear;      /* wedge clearance angle (rad) */
    double tool_tip_dz;     /* tool tip z relative to the reference point */
    double newton_tol;      /* relative residual for the Newton return */
    int32_t newton_maxit;
    /* particle-side tool contact after every contact_every-th step (0: off),
     * xpbdContactSDFKernel (src/ContactSolver.cu:797-923) on the analytic SDF */
    int32_t contact_every;
    double contact_radius, contact_friction, contact_heat_partition;
    /* adiabatic shear band heating after g2p (asb_enabled != 0), restating
     * applyAdiabaticHeatingKernel (src/AdiabaticShearModel.cu:104-177); the
     * heated-particle guard is T > Tamb + asb_touch_rise */
    int32_t asb_enabled;
    double asb_critical_rate, asb_taylor_quinney, asb_max_temp_ratio, asb_touch_rise;
    /* grid heat conduction (heat_conduction != 0) as MPMWorkpieceSolver does
     * it: T m scattered with the mass, one explicit diffusion step on the grid
     * (mpmDiffuseTemperatureKernel, src/MPMWorkpieceSolver.cu:208-262), T
     * gathered back in g2p (:282-306); alpha = k / (rho_phys cp) */
    int32_t heat_conduction;
    double thermal_conductivity;
    /* voxel tool SDF for the contact (NULL: the analytic SDF): its frame's
     * origin follows the tool reference point, rotated by tool_sdf_angle
     * about z; the contact then is xpbdContactSDFKernel's (orc_contact_sdf) */
    const struct orc_sdf_grid *tool_sdf;
    float tool_sdf_angle;
} orc_params;

/* Particle state, SoA, one entry per particle (matrices row-major [n][9],
 * symmetric tensors [n][6] as xx,yy,zz,xy,xz,yz). */
typedef struct orc_state {
    int32_t n;
    int32_t _pad;
    double *x, *y, *z;
    double *vx, *vy, *vz;
    double *F, *Fp, *C;
    double *sig, *bs;
    double *eps, *edot, *T, *D, *sres;
    double *mass, *vol;
    double *extf;            /* [n][3] or NULL: applied for one step, then zeroed */
    int32_t *status, *id;
    int32_t *lod;            /* [n] LOD zone, persists like MPMParticle::lodZone */
    int32_t *asb;            /* [n] or NULL: adiabatic shear counter, MPMParticle::asbCounter */
} orc_state;

/* Rasterised tool samples: offsets from the tool reference point. */
typedef struct orc_tool_samples {
    int32_t n;
    int32_t _pad;
    const double *ox, *oy, *oz;
} orc_tool_samples;

/* Conservation and reference-compatible metrics (all FP64). */
typedef struct orc_metrics {
    double mass, px, py, pz, kinetic, internal_elastic, thermal;
    double max_T, max_vm, max_eps, sum_eps;
    double ref_max_stress, ref_max_T, ref_kinetic, ref_internal;
    int64_t n_active, n_chip, n_fixed, n_inactive;
    double bmin[3], bmax[3];
} orc_metrics;

/* One pass of the adiabatic shear heating (applyAdiabaticHeatingKernel) over
 * the particles, as orc_step runs it after g2p when asb_enabled is set; needs
 * s->asb. */
void orc_asb_heat(const orc_params *p, orc_state *s, double dt);

/* One diffusion step on node arrays of nx*ny*nz doubles (mass, T m) -> the
 * node temperatures, as orc_step runs it between the grid update and g2p. */
void orc_heat_diffuse(const orc_params *p, const double *mass, const double *tm, double *tn, double dt);

/* A voxel signed-distance grid of the tool (ToolSDF, src/ToolSDF.cu):
 * v[ix + nx (iy + ny iz)] is the distance at the centre of voxel (ix,iy,iz),
 * o + (i + 1/2) voxel, negative inside the tool. */
typedef struct orc_sdf_grid {
    int32_t nx, ny, nz;
    int32_t _pad;
    const float *v;
    float ox, oy, oz, voxel;
} orc_sdf_grid;

/* Arguments of xpbdContactSDFKernel (src/ContactSolver.cu:797-813): the tool
 * transform (world -> SDF rest frame: translate by -c, rotate by -angle about
 * z), contact radius, friction, heat partition, dt, and the workpiece's
 * specific heat, physical density and melting temperature. */
typedef struct orc_contact_sdf_args {
    float cx, cy, cz, cos_a, sin_a;
    float radius, friction, heat_partition, dt;
    float _pad;
    double cp, rho_phys, Tm;
} orc_contact_sdf_args;

/* A 3D float texture fetch with trilinear filtering, clamp addressing and
 * unnormalised coordinates, as the texture unit computes it (the weights are
 * held with 8 fractional bits; the exact split is in mpm_oracle.c). */
float orc_tex3d(const orc_sdf_grid *g, float x, float y, float z);

/* One pass of xpbdContactSDFKernel over the particles (not INACTIVE or
 * FIXED); count, friction work and normal force summed as its metrics. */
void orc_contact_sdf(const orc_sdf_grid *g, const orc_contact_sdf_args *a, orc_state *s, int64_t *count,
                     double *heat, double *force);

/* The voxel SDF of a closed triangle mesh as ToolSDF builds it
 * (src/ToolSDF.cu:212-280 build, :348-377 buildFromVerts, :379-532
 * computeSDFCPU): verts [nv][3], tris [nt][3] indices, normals [nt][3]
 * (the mesh's triangle normals).  Always fills dims, origin and voxel; fills
 * values (dims product, x fastest) when values is not NULL.  Returns 0, or -1
 * for an empty mesh or grid. */
int orc_tool_sdf_build(const float *verts, int32_t nv, const int32_t *tris, int32_t nt, const float *normals,
                       double padding, int32_t voxels_per_axis, int32_t dims[3], float origin[3], float *voxel,
                       float *values);

/* Size in doubles of the grid scratch that orc_step needs. */
int64_t orc_grid_doubles(const orc_params *p);

/* Advance `nsteps` steps of size dt.  step0 is the solver's step counter
 * before the first step (chip separation runs when the counter is a
 * multiple of chip_every) and t0 the simulation time.  grid is scratch of
 * orc_grid_doubles() doubles.  Returns 0, or a nonzero error code (1: a
 * Newton return did not converge). */
int orc_step(const orc_params *p, orc_state *s, const orc_tool_samples *tool,
             double *grid, double dt, int32_t nsteps, int64_t step0, double t0,
             int32_t nthreads);

/* The other MPM solver of the reference, MPMWorkpieceSolver
 * (src/MPMWorkpieceSolver.cu), which the engine never constructs: trilinear
 * PIC transfers, a hypoelastic stress rate with a Johnson-Cook radial return
 * at the old plastic strain, and a tool boundary that projects out the
 * approaching normal velocity at the nearest tool sample.  Its own constants
 * (MPMMaterialParams, include/MPMWorkpieceSolver.cuh:60-83) beside orc_params,
 * which gives the grid, E and nu (shear and bulk moduli), rho_phys (its
 * density), cp, Tm, Tamb (its reference temperature), A, B, n, C, m, edot0,
 * Dth, Hkin, the fixture thickness and the thermal conductivity. */
typedef struct orc_ws_params {
    double failure_strain;           /* damage += eqRate dt / max(failure_strain, 1e-3) */
    double critical_plastic_strain;  /* ACTIVE -> CHIP at eps >= this */
    double thermal_chip_ratio;       /* ACTIVE -> CHIP at T >= ratio * Tm */
    double tool_contact_radius;      /* a node within this of a tool sample is in contact */
    double contact_damping;          /* heating of a contact: 0.5 m vn^2 * damping */
    double max_contact_temp_rise;    /* per-step cap of contact and plastic heating (thermal clamp) */
    int32_t thermal_clamp;
    int32_t _pad;
} orc_ws_params;

/* Node arrays of one MPMWorkpieceSolver step, for the contact force it sums:
 * *contact_force (may be NULL) receives the last step's sum of
 * |m vn / dt| over the contact nodes (mpmGridUpdateKernel's totalContactForce). */
int64_t orc_ws_grid_doubles(const orc_params *p);

/* Advance nsteps steps of MPMWorkpieceSolver::step (src/MPMWorkpieceSolver.cu:
 * 727-781) on the fixed grid of p: clear, mpmP2GKernel, mpmGridUpdateKernel
 * with the tool samples at pose p0 + v t (offsets in tool), the diffusion
 * step when k / (rho cp) > 0 (Jacobi, as orc_heat_diffuse), mpmG2PKernel, and
 * on even step counts its chipFractureAndSeparationKernel with the tool tip
 * z = pose z + tool_tip_dz.  s->extf, when set, is the particles' force
 * (MPMParticleGPU::f), applied in the first step and then zeroed as
 * mpmG2PKernel does; s->bs is the backstress. */
void orc_ws_step(const orc_params *p, const orc_ws_params *w, orc_state *s, const orc_tool_samples *tool, double *grid,
                 double dt, int32_t nsteps, int64_t step0, double t0, double *contact_force);

/* Tool SDF at a world point for the tool reference point pr. */
double orc_tool_sdf(const orc_params *p, const double pr[3], double x, double y, double z);

void orc_metrics_compute(const orc_params *p, const orc_state *s, orc_metrics *out);

/* Philox4x32-10 (Salmon et al., SC'11): 4 uniform floats in [0,1) per call,
 * 24-bit resolution.  Used by the seeded workpiece generator. */
void orc_philox_uniform4(uint32_t seed_lo, uint32_t seed_hi, uint32_t c0, uint32_t c1,
                         uint32_t c2, uint32_t c3, float out[4]);

#ifdef __cplusplus
}
#endif
#endif
