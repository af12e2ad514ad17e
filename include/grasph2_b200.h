/*
 * grasph2_b200.h -- C-ABI of the B200 (sm_100a) implementation of GraSPH2's per-step hot path:
 * all-pairs self-gravity with Plummer softening, the SPH density sum, the stress/pressure
 * acceleration with artificial viscosity, the Jaumann stress rate, the plasticity limiter and the
 * leapfrog integrator.
 *
 * Plain C: fixed-width integers, plain pointers and sizes. No CUDA or C++ types appear in the
 * signatures; a stream is passed as `void*` (a cudaStream_t, or NULL for the legacy default
 * stream). Every entry point returns an int status: 0 on success, a negative GSPH_E_* code on
 * failure. The text of the last failure on a context is available from gsph_last_error().
 *
 * Reference surface this replaces (GraSPH2 source tree):
 *   - compile-time switches and constants   settings/settings.h:26-185
 *   - precision types f1_t/f3_t/m3_t        settings/precisionSettings.h:16-17, src/types.h:32-56
 *   - particle attributes, in this order    src/particles/partice_attributes.h:91-106
 *   - DeviceParticleBuffer (owning buffers) src/particles/DeviceParticleBuffer.h:47-233,
 *                                           src/particles/Device_base.h:126-203
 *   - computeDerivatives(pb)                src/computeDerivatives.h:315-328
 *   - integrate(pb, notFirstStep)           src/integration.h:219-244
 *   - getCurrentTimestep()                  src/integration.h:246-255
 *
 * One context = one simulation (or one ensemble) on the current CUDA device. Calls on one
 * context are not thread-safe; distinct contexts may be driven from distinct host threads.
 */
#ifndef GRASPH2_B200_H
#define GRASPH2_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GSPH_ABI_VERSION 1

/* ---------------------------------------------------------------------------------------------
 * status codes
 * ------------------------------------------------------------------------------------------- */
#define GSPH_OK              0
#define GSPH_E_INVALID     (-1)  /* bad argument: null pointer, size out of range, bad mask/flags */
#define GSPH_E_CUDA        (-2)  /* a CUDA runtime call or a kernel launch failed */
#define GSPH_E_NOMEM       (-3)  /* device or pinned host allocation failed */
#define GSPH_E_STATE       (-4)  /* call not valid in the context's current state */
#define GSPH_E_NUMERIC     (-5)  /* non-finite values found by a host-requested scan */
#define GSPH_E_TIMEOUT     (-6)  /* a bounded device-side wait gave up (status word set) */
#define GSPH_E_UNSUPPORTED (-7)  /* feature combination not implemented */

/* ---------------------------------------------------------------------------------------------
 * physics switches: one bit per `#define` of settings/settings.h
 * ------------------------------------------------------------------------------------------- */
#define GSPH_SELF_GRAVITY          (1u << 0)   /* ENABLE_SELF_GRAVITY         settings.h:34  */
#define GSPH_SPH                   (1u << 1)   /* ENABLE_SPH                  settings.h:37  */
#define GSPH_INTEGRATE_DENSITY     (1u << 2)   /* INTEGRATE_DENSITY           settings.h:40  */
#define GSPH_DEAL_WITH_NO_PARTNERS (1u << 3)   /* DEAL_WITH_NO_PARTNERS       settings.h:41  */
#define GSPH_SOLIDS                (1u << 4)   /* SOLIDS                      settings.h:42  */
#define GSPH_VARIABLE_TIMESTEP     (1u << 5)   /* VARIABLE_TIMESTEP_LEAPFROG  settings.h:55 (off: FIXED_TIMESTEP_LEAPFROG :49) */
#define GSPH_ACCELERATION_CRITERION (1u << 6)  /* ACCELERATION_CRITERION      settings.h:59  */
#define GSPH_VELOCITY_CRITERION    (1u << 7)   /* VELOCITY_CRITERION          settings.h:61  */
#define GSPH_PLASTICITY_MIESE      (1u << 8)   /* PLASTICITY_MIESE            settings.h:116 */
#define GSPH_PLASTICITY_MC         (1u << 9)   /* PLASTICITY_MC               settings.h:120 */
#define GSPH_CLOHESSY_WILTSHIRE    (1u << 10)  /* CLOHESSY_WILTSHIRE          settings.h:136 */
#define GSPH_CONSTANT_ACCELERATION (1u << 11)  /* CONSTANT_ACCELERATION       settings.h:141 */
#define GSPH_SIMPLE_BOX_BOUNDARY   (1u << 12)  /* SIMPLE_BOX_BOUNDARY         settings.h:146 */
#define GSPH_ARTIFICIAL_VISCOSITY  (1u << 13)  /* ARTIFICIAL_VISCOSITY        settings.h:155 */
#define GSPH_BALSARA_SWITCH        (1u << 14)  /* BALSARA_SWITCH              settings.h:159 */
#define GSPH_ARTIFICIAL_STRESS     (1u << 15)  /* ARTIFICIAL_STRESS           settings.h:163 */
#define GSPH_XSPH                  (1u << 16)  /* XSPH                        settings.h:170 */
#define GSPH_ALL_FLAGS             ((1u << 17) - 1u)

/* ---------------------------------------------------------------------------------------------
 * runtime parameters: the `constexpr` values of settings/settings.h, plus two knobs the
 * reference hard-wires (grav_eps, av_beta). Doubles on the host; the kernels round them to the
 * arithmetic type they compute in.
 * ------------------------------------------------------------------------------------------- */
typedef struct gsph_params {
    uint32_t flags;            /* GSPH_* switches above */
    int32_t  dimension;        /* 1, 2 or 3                                   settings.h:31      */
    double   H;                /* smoothing length; kernel support radius   settings.h:99      */
    double   grav_eps;         /* Plummer softening; the reference uses eps == H
                                  (src/computeDerivatives.h:231)                                  */
    double   grav_G;           /* gravitational constant; the reference uses 1                    */
    double   rho0;             /* rest density                               settings.h:105     */
    double   bulk;             /* bulk modulus K0 (Murnaghan)                settings.h:106     */
    double   dbulk_dp;         /* dK0/dP (Murnaghan exponent)                settings.h:107     */
    double   soundspeed;       /* c: liquid EOS c^2 and AV signal speed      settings.h:108     */
    double   shear;            /* shear modulus mu                           settings.h:111     */
    double   Y;                /* von Mises yield stress                     settings.h:117     */
    double   tanfr;            /* tan(friction angle), Mohr-Coulomb          settings.h:122     */
    double   cohesion;         /* Mohr-Coulomb cohesion                      settings.h:123     */
    double   av_alpha;         /* artificial viscosity strength              settings.h:156     */
    double   av_beta;          /* AV signal velocity v_sig = c_i + c_j - av_beta * w; the
                                  reference fixes av_beta = 3 (src/sph/models.h:179)             */
    double   mateps;           /* artificial stress strength                 settings.h:164     */
    double   matexp;           /* artificial stress exponent                 settings.h:165     */
    double   normalsep;        /* artificial stress reference separation     settings.h:166     */
    double   xsph_factor;      /* XSPH velocity smoothing factor             settings.h:171     */
    double   fixed_dt;         /* fixed leapfrog step                        settings.h:50      */
    double   initial_dt;       /* variable leapfrog: first step              settings.h:56      */
    double   min_dt;           /*                    lower clamp             settings.h:57      */
    double   max_dt;           /*                    upper clamp             settings.h:58      */
    double   accel_accuracy;   /* dt <= sqrt(accel_accuracy * H / |a|)       settings.h:60      */
    double   velocity_accuracy;/* dt <= velocity_accuracy * H / v_sig,max    settings.h:62      */
    double   cw_n;             /* Clohessy-Wiltshire mean motion n           settings.h:137     */
    double   const_acc[3];     /* constant acceleration                      settings.h:142     */
    double   box_min[3];       /* simple box boundary                        settings.h:147     */
    double   box_max[3];       /*                                            settings.h:148     */
    double   box_reflectiveness; /*                                          settings.h:149     */
} gsph_params;

/* Fill `p` with the values of the reference's shipped settings/settings.h (a rotating solid
 * sphere with Mohr-Coulomb plasticity, variable time step, AV and the Balsara switch). */
int gsph_params_reference_defaults(gsph_params* p);

/* Check a parameter set; returns GSPH_OK or GSPH_E_INVALID / GSPH_E_UNSUPPORTED and, when
 * `msg`/`msg_len` are given, a one-line reason. */
int gsph_params_validate(const gsph_params* p, char* msg, size_t msg_len);

/* ---------------------------------------------------------------------------------------------
 * particle attributes: bit order = particle_bases (src/particles/partice_attributes.h:106)
 * ------------------------------------------------------------------------------------------- */
#define GSPH_POS        (1u << 0)   /* f3  */
#define GSPH_MASS       (1u << 1)   /* f1  */
#define GSPH_VEL        (1u << 2)   /* f3  */
#define GSPH_ACC        (1u << 3)   /* f3  */
#define GSPH_BALSARA    (1u << 4)   /* f1  */
#define GSPH_XVEL       (1u << 5)   /* f3  */
#define GSPH_DENSITY    (1u << 6)   /* f1  */
#define GSPH_DENSITY_DT (1u << 7)   /* f1  */
#define GSPH_DSTRESS    (1u << 8)   /* m3: 9 values, row-major (tsv/h5 order, src/ResultStorageManager.cu:141-149) */
#define GSPH_DSTRESS_DT (1u << 9)   /* m3 */
#define GSPH_MAXVSIG    (1u << 10)  /* f1  */
#define GSPH_ALL_ATTRIBS ((1u << 11) - 1u)

/* Host-side particle data in the reference's attribute layout (array-of-structs per attribute,
 * i.e. pos = x0,y0,z0,x1,...). Only the pointers whose bit is set in the call's mask are read or
 * written; the others may be NULL. Single precision, as f1_t with SINGLE_PRECISION. */
typedef struct gsph_host_particles {
    float* pos;        /* 3N */
    float* mass;       /* N  */
    float* vel;        /* 3N */
    float* acc;        /* 3N */
    float* balsara;    /* N  */
    float* xvel;       /* 3N */
    float* density;    /* N  */
    float* density_dt; /* N  */
    float* dstress;    /* 9N */
    float* dstress_dt; /* 9N */
    float* maxvsig;    /* N  */
} gsph_host_particles;

/* ---------------------------------------------------------------------------------------------
 * numerics and launch options of a context
 * ------------------------------------------------------------------------------------------- */
#define GSPH_ACCUM_PLAIN       0  /* FP32 accumulation throughout the pair sums */
#define GSPH_ACCUM_COMPENSATED 1  /* FP32 within a j-tile, two-sum (Kahan-Babuska) fold of each
                                     tile's partial into the running sum, FP64 combine of j-splits */

typedef struct gsph_options {
    int32_t accum;           /* GSPH_ACCUM_* */
    int32_t j_split;         /* j-segments per i-block (0 = pick from N and the SM count) */
    int32_t j_tile;          /* j-particles per shared-memory stage (0 = default) */
    int32_t i_per_thread;    /* register blocking of the gravity-only kernel: 1, 2, 4 or 8 (0 = default) */
    int32_t threads;         /* threads per CTA of the pair kernels (0 = default) */
    int32_t check_finite;    /* nonzero: scan inputs at upload for NaN/Inf and fail with GSPH_E_NUMERIC */
    int32_t no_cull;         /* 0 (default): particles are kept in Hilbert-curve order on the device and the SPH
                                passes visit only chunks within H of each particle group, gravity covering
                                all pairs in its own kernel; nonzero: every SPH pass sweeps all N^2 pairs */
    int32_t resort_interval; /* re-sort the curve order every this many gsph_step steps (0: only when
                                positions are uploaded) */
    int32_t scalar_fp32;     /* nonzero: scalar FP32 gravity kernel instead of the paired f32x2 form
                                (identical results; for comparison) */
    int32_t precision;       /* GSPH_PRECISION_SINGLE (default) or GSPH_PRECISION_DOUBLE: the reference's
                                SINGLE_PRECISION / DOUBLE_PRECISION switch (settings/precisionSettings.h:16-17).
                                Double runs every pass in FP64 with plain all-pairs tiles (no culling,
                                accum ignored); gsph_upload_f64 / gsph_download_f64 pass values unrounded */
    int32_t gravity_form;    /* GSPH_GRAVITY_AUTO (default), GSPH_GRAVITY_ONE_SIDED or GSPH_GRAVITY_SYMMETRIC: the
                                all-pairs gravity kernel evaluates every ordered pair (i gathers from all j), or
                                every unordered pair once and applies it to both particles (Newton's third law;
                                2/3 of the FP32 work, partials of 65 x 3 floats per particle). Auto picks the
                                symmetric form from 24 blocks of 1024 particles up. Results agree to rounding.
                                Ensembles use the one-sided sweep fused with their density pass; SYMMETRIC
                                gives them a queue stage of group pairs instead (slower on ensembles of
                                1k..32k-particle simulations) */
    int32_t gravity_groups;  /* symmetric form: particle groups G (tasks G(G+1)/2); 0 = up to 64 */
    int32_t wait_limit_us;   /* batched ensemble: a work item that waits for another item's result (a device-side
                                spin on a counter) gives up after this many microseconds, sets the timeout bit
                                and its call returns GSPH_E_TIMEOUT (0 = 2 s). Waits for a bulk copy to land
                                keep the fixed 2 s bound */
    int32_t reserved[3];
} gsph_options;

#define GSPH_PRECISION_SINGLE 0
#define GSPH_PRECISION_DOUBLE 1
#define GSPH_GRAVITY_AUTO      0
#define GSPH_GRAVITY_ONE_SIDED 1
#define GSPH_GRAVITY_SYMMETRIC 2

int gsph_options_defaults(gsph_options* o);

typedef struct gsph_ctx gsph_ctx;

/* Create a simulation of n particles on the current device with parameters `p` (copied).
 * Allocates the device attribute buffers (the analogue of DeviceParticleBuffer's constructor,
 * src/particles/Device_base.h:126-145). `opt` may be NULL for defaults. */
int gsph_create(const gsph_params* p, const gsph_options* opt, int64_t n, gsph_ctx** out);
int gsph_destroy(gsph_ctx* ctx);

/* Copy host attributes -> device (pb = hostBuffer, src/particles/Device_base.h:163-181).
 * `attr_mask` picks the attributes; DSTRESS is symmetrised on upload (the kernels store the six
 * independent components). Positions are also kept as an FP64 master copy on the device. The
 * device may hold the particles in another order (see gsph_options.no_cull); every transfer uses the
 * caller's order. */
int gsph_upload(gsph_ctx* ctx, uint32_t attr_mask, const gsph_host_particles* src, void* stream);
/* Copy device -> host for the attributes in `attr_mask`; synchronises `stream`. */
int gsph_download(gsph_ctx* ctx, uint32_t attr_mask, gsph_host_particles* dst, void* stream);
/* The same transfers in double precision: the host buffers of the reference's DOUBLE_PRECISION build
 * (src/types.h:32-43, f1_t = double). With GSPH_PRECISION_DOUBLE the values pass unrounded; in single
 * precision they are rounded to float on upload and widened on download. */
typedef struct gsph_host_particles64 {
    double* pos;        /* 3N */
    double* mass;       /* N  */
    double* vel;        /* 3N */
    double* acc;        /* 3N */
    double* balsara;    /* N  */
    double* xvel;       /* 3N */
    double* density;    /* N  */
    double* density_dt; /* N  */
    double* dstress;    /* 9N */
    double* dstress_dt; /* 9N */
    double* maxvsig;    /* N  */
} gsph_host_particles64;
int gsph_upload_f64(gsph_ctx* ctx, uint32_t attr_mask, const gsph_host_particles64* src, void* stream);
int gsph_download_f64(gsph_ctx* ctx, uint32_t attr_mask, gsph_host_particles64* dst, void* stream);

/* FP64 positions (3N, x0,y0,z0,...): upload overrides the FP32 positions; download reads the master. */
int gsph_upload_pos64(gsph_ctx* ctx, const double* pos, void* stream);
int gsph_download_pos64(gsph_ctx* ctx, double* pos, void* stream);

/* computeDerivatives(pb)  -- src/computeDerivatives.h:315-328.
 * Density sum (unless INTEGRATE_DENSITY), then one fused all-pairs pass for gravity, stress
 * acceleration, AV, strain/rotation rates and the Jaumann stress rate. With the Balsara switch
 * on, the velocity-gradient pass runs first as its own pass (the reference's
 * calcBalsaraDensityDTDStressDT), since the acceleration needs every B_j. Asynchronous. */
int gsph_compute_derivatives(gsph_ctx* ctx, void* stream);

/* integrate(pb, notFirstStep) -- src/integration.h:219-244. Fixed or variable leapfrog with
 * density/stress update, plasticity and boundaries. The variable step keeps dt on the device
 * (no host synchronisation). Asynchronous. */
int gsph_integrate(gsph_ctx* ctx, int not_first_step, void* stream);

/* nsteps x { computeDerivatives; integrate(notFirstStep = true) } -- the loop of
 * src/main.cu:249-273 without I/O. The step is captured once into a CUDA graph and replayed. */
int gsph_step(gsph_ctx* ctx, int32_t nsteps, void* stream);

/* getCurrentTimestep() -- src/integration.h:246-255: the fixed step, or the last variable step
 * (synchronises `stream`). */
int gsph_current_timestep(gsph_ctx* ctx, double* dt, void* stream);

/* FP64 diagnostics of the current state (no reference counterpart: the reference has none). */
typedef struct gsph_diag {
    double e_kin;        /* 1/2 sum m v^2 (v as stored)                      */
    double e_grav;       /* -G sum_{i<j} m_i m_j / sqrt(r^2 + eps^2)          */
    double e_int;        /* sum m u(rho), barotropic u of the EOS             */
    double e_shear;      /* sum m S:S / (4 mu rho) (solids)                   */
    double momentum[3];  /* sum m v                                           */
    double ang_mom[3];   /* sum m x cross v                                   */
    double mass;         /* sum m                                             */
} gsph_diag;
/* The velocity used is v + half_kick * a (a as last computed): pass 0 for the stored velocity, or
 * 0.5*dt right after gsph_compute_derivatives to synchronise the leapfrog's half-step velocity
 * v_{n-1/2} to v_n. Synchronises `stream`. */
int gsph_diagnostics(gsph_ctx* ctx, double half_kick, gsph_diag* out, void* stream);
/* The same with the pair potential summed in FP32 (two-sum across j-tiles, FP64 across particles;
 * relative error of e_grav ~1e-7): one FP32 N^2 sweep instead of an FP64 one, for frequent checks. */
int gsph_diagnostics_fast(gsph_ctx* ctx, double half_kick, gsph_diag* out, void* stream);

/* Autotuner (no counterpart in the reference): times candidate launch shapes on the context's current
 * state and keeps the fastest, `reps` timed launches each (median): the gravity kernel's i-blocking,
 * j-tile and j-split; the culled SPH passes' work-item count, or the all-pairs SPH tile shape. Results
 * change only by summation order. The next gsph_step re-captures its graph. */
int gsph_autotune(gsph_ctx* ctx, int32_t reps, void* stream);
typedef struct gsph_launch_shape {
    int32_t cull, grav_ipt, grav_jt, grav_nseg, grav_x2, sph_threads, sph_jt, sph_nseg, items;
    int32_t grav_sym_groups;  /* > 0: the symmetric gravity kernel over this many particle groups */
    int32_t reserved[6];
} gsph_launch_shape;
int gsph_launch_shape_get(gsph_ctx* ctx, gsph_launch_shape* out);

/* Number of particles of the context. */
int gsph_size(gsph_ctx* ctx, int64_t* n);
/* Re-sort the device-side particle order along a Hilbert curve of the current positions (a no-op
 * with no_cull set). Results do not depend on the order except for floating-point summation order. */
int gsph_reorder(gsph_ctx* ctx, void* stream);
/* Text of the last failure on `ctx` (or of the last failed gsph_create when ctx is NULL). */
const char* gsph_last_error(gsph_ctx* ctx);
/* Device pointers of the resident arrays, for zero-copy callers (read-only view). */
typedef struct gsph_device_view {
    int64_t n;
    void* posm;      /* float4 x,y,z,m */
    void* velrho;    /* float4 vx,vy,vz,rho */
    void* acc;       /* float4 ax,ay,az,max_vsig */
    void* pos64;     /* double[3][n] (SoA) */
} gsph_device_view;
int gsph_device_view_get(gsph_ctx* ctx, gsph_device_view* v);

/* Number of kernels this context launched since creation (host-side count). */
int gsph_launch_count(gsph_ctx* ctx, int64_t* count);

/* Tensor-core tile GEMM check (no counterpart in the reference): D[128][N] = A[128][K] * B[N][K]^T
 * with bf16 row-major device inputs and FP32 output, each operand staged K-major (0) or MN-major (1)
 * in shared memory as the surrogate's MLP kernels stage theirs. N, K multiples of 16 in [16, 128].
 * Synchronises the device. */
int gsph_tc_gemm_check(const void* A, const void* B, float* D, int32_t N, int32_t K, int32_t a_mn, int32_t b_mn);

/* ---------------------------------------------------------------------------------------------
 * the learned surrogate's per-particle MLP (no counterpart in the reference): 32 inputs, three
 * hidden layers of 128 with SiLU, 13 outputs; BF16 weights and activations on the tensor cores with
 * FP32 accumulation, FP32 master parameters and Adam state on the device. Parameters are one flat
 * FP32 vector: W1[128][32] b1[128] W2[128][128] b2[128] W3[128][128] b3[128] W4[13][128] b4[13].
 * ------------------------------------------------------------------------------------------- */
#define GSPH_MLP_IN  32
#define GSPH_MLP_OUT 13
typedef struct gsph_mlp gsph_mlp;
int64_t gsph_mlp_param_count(void);
/* params: host FP32 vector of gsph_mlp_param_count() values, or NULL for zeros */
int gsph_mlp_create(const float* params, gsph_mlp** out);
int gsph_mlp_destroy(gsph_mlp* m);
int gsph_mlp_get_params(gsph_mlp* m, float* params);
/* replaces the parameters and clears the Adam state */
int gsph_mlp_set_params(gsph_mlp* m, const float* params);
/* y[n][13] = MLP(x[n][32]); device pointers, asynchronous on `stream` */
int gsph_mlp_forward(gsph_mlp* m, const float* x, float* y, int64_t n, void* stream);
/* gradient of L = (1/n) sum_p sum_o wout[o] (y_po - target_po)^2 over the n device rows into the
 * model's gradient buffer (deterministic); grad (host, param_count) and loss (host) may be NULL, else
 * they are filled and `stream` synchronised. wout: 13 device floats */
int gsph_mlp_gradient(gsph_mlp* m, const float* x, const float* target, const float* wout, int64_t n, float* grad,
                      double* loss, void* stream);
/* one Adam step (Kingma & Ba 2015) with the last gradient */
int gsph_mlp_adam(gsph_mlp* m, float lr, float beta1, float beta2, float eps, void* stream);
/* global-norm gradient clipping of the following Adam steps: the gradient is scaled by
 * min(1, max_norm / ||g||_2) first (0 = off, the default) */
int gsph_mlp_set_grad_clip(gsph_mlp* m, float max_norm);
const char* gsph_mlp_last_error(const gsph_mlp* m);

/* Surrogate support on a context (no counterpart in the reference).
 * gsph_surrogate_features: 32 neighbour-moment features of the current state per particle into
 *   feat[n][32] (device, caller's order), standardised as (f - mu) / sigma when mu and sigma (32 device
 *   floats each) are given. Needs SPH in single precision with culling.
 * gsph_surrogate_apply: advance the state by a K-substep proposal: the fixed-step leapfrog with the
 *   derivatives of the last gsph_compute_derivatives held constant, plus out_mu + out_sigma * delta
 *   per particle (delta[n][13] device, caller's order: position 3, velocity 3, density, stress xx yy
 *   zz xy xz yz; NULL for the extrapolation alone), then the plasticity limiter.
 * gsph_snapshot: save (restore = 0) or restore (restore = 1) the whole device state in slot 0..3. */
int gsph_surrogate_features(gsph_ctx* ctx, const float* mu, const float* sigma, float* feat, void* stream);
int gsph_surrogate_apply(gsph_ctx* ctx, const float* delta, const float* out_mu, const float* out_sigma, int32_t K,
                         void* stream);
int gsph_snapshot(gsph_ctx* ctx, int32_t slot, int32_t restore, void* stream);
/* O(N) comparison of the current state Q with the states saved in slot_p (P) and slot_0 (X0), for the
 * surrogate's judge (synchronises `stream`): out[0] = E(P) - E(Q), with the kinetic, internal and shear
 * energies exact and the gravitational energy to first order in x_P - x_Q (-sum m g . dx, g the
 * gravitational acceleration of Q's last derivative evaluation); out[1] = sum |x_P - x_Q|^2;
 * out[2] = sum |x_Q - x_0|^2; out[3] = E_kin + E_int + E_shear of Q. */
int gsph_state_compare(gsph_ctx* ctx, int32_t slot_p, int32_t slot_0, double* out, void* stream);
/* The same with out[4..7] = the parts of out[0]: kinetic, internal, shear, and first-order
 * gravitational energy of P minus Q. */
int gsph_state_compare_parts(gsph_ctx* ctx, int32_t slot_p, int32_t slot_0, double* out, void* stream);
/* Change the kinetic energy about the centre of mass by d_kin and the shear energy by d_shear (no
 * counterpart in the reference; the surrogate's energy correction): peculiar velocities are scaled
 * about the centre-of-mass velocity and the deviatoric stress is scaled (each factor limited to
 * [0.9, 1.1]), then the plasticity limiter of the integrator runs. Momentum and positions are
 * unchanged. Asynchronous on `stream` (three launches). */
int gsph_energy_adjust(gsph_ctx* ctx, double d_kin, double d_shear, void* stream);

/* The learned surrogate as a native object (no counterpart in the reference): its MLP, the
 * standardisation of the 32 inputs and 13 outputs, and K. A proposal advances a context by K substeps
 * at once: gsph_compute_derivatives, gsph_surrogate_features (standardised), gsph_mlp_forward and
 * gsph_surrogate_apply (use_net = 0: the extrapolation alone). A window is M proposals whose last one
 * the plain integrator re-advances from the same state as judge; it is accepted when the proposal is
 * within pos_tol of the plain result in position (norm over all particles, relative to the plain
 * displacement) and within e_tol in total energy (relative to the energy at the start of the
 * gsph_surrogate_advance call), and the state continues from the plain result; otherwise the window is
 * re-run by the plain integrator from its start. Uses snapshot slots 0-2 of the context and
 * synchronises `stream` once per window. Statistics (create's scale arrays; NULL means 0 for a mean and
 * 1 for a sigma) and the model file hold, in order, in_mu[32], in_sigma[32], out_mu[13], out_sigma[13].
 * Model file (little-endian): "GSPHSUR1", int32 K, int32 parameter count, the FP32 parameters, the 90
 * FP32 statistics. */
typedef struct gsph_surrogate gsph_surrogate;
typedef struct gsph_surrogate_window {
    double pos_error;        /* ||x_proposal - x_plain||_2 / ||x_plain - x_start||_2 of the judged proposal */
    double energy_error;     /* |E_proposal - E_plain| / |E_ref|                                        */
    double energy_parts[4];  /* signed (E_proposal - E_plain) / |E_ref|: kinetic, internal, shear,
                                gravitational (first order)                                             */
    int32_t accepted;
    int32_t reserved;
} gsph_surrogate_window;
#define GSPH_SURROGATE_STATS 90
int gsph_surrogate_create(const float* params, const float* in_mu, const float* in_sigma, const float* out_mu,
                          const float* out_sigma, int32_t K, gsph_surrogate** out);
int gsph_surrogate_load(const char* path, gsph_surrogate** out);
int gsph_surrogate_save(gsph_surrogate* s, const char* path);
int gsph_surrogate_destroy(gsph_surrogate* s);
/* the surrogate's own MLP (owned by it), e.g. to train it with gsph_mlp_gradient / gsph_mlp_adam */
gsph_mlp* gsph_surrogate_mlp(gsph_surrogate* s);
int32_t gsph_surrogate_substeps(const gsph_surrogate* s);
/* the GSPH_SURROGATE_STATS statistics into stats (host) */
int gsph_surrogate_stats(const gsph_surrogate* s, float* stats);
int gsph_surrogate_propose(gsph_surrogate* s, gsph_ctx* ctx, int32_t use_net, void* stream);
/* one judged proposal from the current state; the context ends on the plain result. e_ref: the energy
 * scale of out->energy_error, or 0 for the current total energy (gsph_diagnostics_fast) */
int gsph_surrogate_judge(gsph_surrogate* s, gsph_ctx* ctx, int32_t use_net, double e_ref, gsph_surrogate_window* out,
                         void* stream);
/* nwin windows; windows (nwin entries) and accepted may be NULL */
int gsph_surrogate_advance(gsph_surrogate* s, gsph_ctx* ctx, int32_t nwin, int32_t M, double pos_tol, double e_tol,
                           int32_t use_net, gsph_surrogate_window* windows, int32_t* accepted, void* stream);
/* Energy correction calibrated by the judge (off by default). An MSE-trained network loses a little
 * kinetic and shear energy in every proposal, the same way each time, which adds up over many windows
 * although each judged proposal passes. With it on, every proposal is followed by
 * gsph_energy_adjust(ctx, -b_kin, -b_shear) with the surrogate's running estimates b of one proposal's
 * bias, and every judged window whose position error is within pos_tol updates them from the judge's
 * comparison: b += gain * (E_proposal - E_plain) of each part (the judged proposal is corrected too, so
 * that is the residual). gain in (0, 1]; setting resets the estimates to zero. */
int gsph_surrogate_set_energy_correction(gsph_surrogate* s, int32_t on, double gain);
/* bias[2]: the current estimates (kinetic, shear; energy units) */
int gsph_surrogate_energy_bias(const gsph_surrogate* s, double* bias);
/* MLP forward launches made by the surrogate (the context counts its own kernels) */
int gsph_surrogate_launch_count(const gsph_surrogate* s, int64_t* count);
const char* gsph_surrogate_last_error(const gsph_surrogate* s);

/* ---------------------------------------------------------------------------------------------
 * initial conditions on the device (the reference's particle sources, src/initialConditions/
 * particleSources/UniformSphere.cu, PlummerSphere.cu, and the centre-of-mass correction of
 * InitGenerator.h:113-152). Outputs are device arrays in the host layout of gsph_host_particles
 * (pos/vel 3n floats), ready for gsph_upload_device. Draws are counter-based (splitmix64 of seed,
 * draw and particle index): independent of the launch shape and reproducible on the host.
 * ------------------------------------------------------------------------------------------- */
int gsph_ic_uniform_sphere(int64_t n, double radius, double total_mass, double rho0, const double* omega,
                           uint64_t seed, float* pos, float* vel, float* mass, float* density, void* stream);
int gsph_ic_plummer(int64_t n, double a, double total_mass, double G, uint64_t seed, float* pos, float* vel,
                    float* mass, void* stream);
/* subtract the mass-weighted mean position and velocity (vel may be NULL); scratch: 7 * 256 device doubles */
int gsph_ic_com_correct(int64_t n, float* pos, float* vel, const float* mass, double* scratch, void* stream);
/* shift positions and/or velocities so that their mass-weighted means become com[3] / vcom[3] (either may
 * be NULL: left as is): the per-source correction of InitGenerator.h:113-152, whose targets are the
 * desired centre of mass and its velocity that gsph_ic_modify tracks; scratch: 7 * 256 device doubles */
int gsph_ic_com_set(int64_t n, float* pos, float* vel, const float* mass, const double* com, const double* vcom,
                    double* scratch, void* stream);

/* Modifiers of a particle source (ParticleSource, src/initialConditions/ParticleSource.h:65-74 and
 * :93-203), applied on the device to every particle in list order, as the reference applies its
 * m_operations to each generated particle. */
#define GSPH_IC_MOVE         1  /* pos += v[0..2]                                          (move)               */
#define GSPH_IC_ROTATE       2  /* pos = R pos, vel = R vel; axis v[0..2], angle v[3] (rad)  (rotate)             */
#define GSPH_IC_POS_NOISE    3  /* pos += three draws uniform in [-v[0], v[0]) from `seed`   (addPositionalNoise) */
#define GSPH_IC_ANGULAR_VEL  4  /* vel += omega x pos, omega = v[0..2]                       (addAngularVelocity) */
#define GSPH_IC_LINEAR_VEL   5  /* vel += v[0..2]                                            (addLinearVelocity)  */
#define GSPH_IC_RANDOM_VEL   6  /* vel += three draws uniform in [-v[0], v[0]) from `seed`   (addRandomVelocity)  */
#define GSPH_IC_SET_CONSTANT 7  /* attribute `attr` (one GSPH_* bit) = v[0..k-1], k its components (setConstant) */
typedef struct gsph_ic_op {
    int32_t kind;   /* GSPH_IC_* */
    uint32_t attr;  /* GSPH_IC_SET_CONSTANT: the attribute bit */
    uint64_t seed;  /* the random modifiers: draw j of particle i is splitmix64-based, (seed, j, i) */
    double v[9];
} gsph_ic_op;
#define GSPH_IC_MAX_OPS 16
/* Apply ops[0..nops-1] (nops <= GSPH_IC_MAX_OPS) to the n particles of `dev` (device arrays in the host
 * layout; an op whose attribute array is NULL fails with GSPH_E_INVALID). desired_com / desired_vcom
 * (host double[3], in/out, may be NULL) are transformed as the reference's m_desiredCOM /
 * m_desiredVelOfCOM: move adds to the COM, rotate rotates both, the velocity modifiers add their
 * (deterministic) part to the COM velocity. The random modifiers draw the reference's distribution
 * (uniform in [-s, s) per component) from counter-based draws instead of std::default_random_engine's
 * sequence, so values are reproducible for any launch shape but not bit-equal to the reference's. */
int gsph_ic_modify(int64_t n, const gsph_ic_op* ops, int32_t nops, const gsph_host_particles* dev,
                   double* desired_com, double* desired_vcom, void* stream);
/* gsph_upload from device arrays in the host layout (e.g. the generators above) */
int gsph_upload_device(gsph_ctx* ctx, uint32_t attr_mask, const gsph_host_particles* src, void* stream);

/* ---------------------------------------------------------------------------------------------
 * asynchronous snapshot output (the reference's ResultStorageManager, src/ResultStorageManager.h:
 * 140-148, .cu:102-186): gsph_writer_write copies the context's state on the device into one of
 * `depth` slots (ordered on `stream`), converts and copies it to pinned host memory on the writer's own
 * stream, and returns; a worker thread writes the tsv file (GraSPH2's format and attribute order).
 * When every slot is busy, write waits for the oldest. Calls on a writer come from the thread that
 * drives its context; the context must outlive the writer.
 * ------------------------------------------------------------------------------------------- */
/* HDF5 snapshots (the reference's STORE_HDF5 output, src/ResultStorageManager.cu:191-227, and its
 * HDF5File particle source, src/initialConditions/particleSources/HDF5File.h:38-150): one float dataset
 * per attribute in `mask`, named POS, MASS, VEL, ACC, BALSARA, XVEL, DENSITY, DENSITY_DT, DSTRESS,
 * DSTRESS_DT, MAXVSIG, of shape {n, components}. The system's libhdf5 (1.10 or later) is loaded when
 * first needed; without it these return GSPH_E_UNSUPPORTED (the reference's HDF5_AVAILABLE check,
 * CMakeLists.txt:123-130). gsph_h5_read: n = the file's particle count; the arrays of `out` selected by
 * `mask` (capacity `cap` particles) receive the values; mask 0 only counts. gsph_writer_write writes
 * HDF5 instead of tsv when the file name ends in ".h5". */
int gsph_h5_available(void);
int gsph_h5_write(const char* filename, int64_t n, const gsph_host_particles* h, uint32_t mask);
int gsph_h5_read(const char* filename, uint32_t mask, gsph_host_particles* out, int64_t cap, int64_t* n);

typedef struct gsph_writer gsph_writer;
int gsph_writer_create(gsph_ctx* ctx, uint32_t attr_mask, int32_t depth, gsph_writer** out);
int gsph_writer_write(gsph_writer* w, const char* filename, void* stream);
/* wait until every queued snapshot is on disk; the first failure's status (message in
 * gsph_writer_last_error), `written` (nullable) = files written so far */
int gsph_writer_flush(gsph_writer* w, int64_t* written);
const char* gsph_writer_last_error(gsph_writer* w);
int gsph_writer_destroy(gsph_writer* w);

/* ---------------------------------------------------------------------------------------------
 * batched ensemble: S independent simulations of uneven particle counts with one parameter set,
 * advanced by one persistent launch per substep. No counterpart in the reference, which runs one
 * simulation per process (src/main.cu:228-273); each simulation follows computeDerivatives /
 * integrate exactly as a single context does (gravity, density and SPH terms only within its own
 * particles). Host arrays hold the simulations back to back: simulation k is rows
 * [offsets[k], offsets[k+1]) with offsets from gsph_ensemble_offsets. Fixed time step, single
 * precision; BALSARA_SWITCH and VARIABLE_TIMESTEP give GSPH_E_UNSUPPORTED.
 * ------------------------------------------------------------------------------------------- */
typedef struct gsph_ensemble gsph_ensemble;
int gsph_ensemble_create(const gsph_params* p, const gsph_options* opt, int32_t nsims, const int64_t* counts,
                         gsph_ensemble** out);
int gsph_ensemble_destroy(gsph_ensemble* e);
/* nsims + 1 row offsets of the packed host layout */
int gsph_ensemble_offsets(const gsph_ensemble* e, int64_t* offsets);
int gsph_ensemble_upload(gsph_ensemble* e, uint32_t attr_mask, const gsph_host_particles* src, void* stream);
/* synchronises `stream` */
int gsph_ensemble_download(gsph_ensemble* e, uint32_t attr_mask, gsph_host_particles* dst, void* stream);
/* FP64 positions (3N) of the master copy, as gsph_upload_pos64 / gsph_download_pos64 */
int gsph_ensemble_upload_pos64(gsph_ensemble* e, const double* pos, void* stream);
int gsph_ensemble_download_pos64(gsph_ensemble* e, double* pos, void* stream);
int gsph_ensemble_compute_derivatives(gsph_ensemble* e, void* stream);
int gsph_ensemble_integrate(gsph_ensemble* e, int32_t not_first_step, void* stream);
/* nsteps x {computeDerivatives; integrate(true)} for every simulation, one captured graph per step */
int gsph_ensemble_step(gsph_ensemble* e, int32_t nsteps, void* stream);
/* FP64 diagnostics of every simulation into out[nsims] (as gsph_diagnostics); synchronises `stream` */
int gsph_ensemble_diagnostics(gsph_ensemble* e, double half_kick, gsph_diag* out, void* stream);
/* Autotuner: times the DENS j-tile (256, 512, 1024) and the CTAs per SM of the persistent grid on the
 * current state (derivative launches only) and keeps the fastest; tile / per_sm (nullable) receive the
 * choice (per_sm 0: as many as fit). */
int gsph_ensemble_autotune(gsph_ensemble* e, int32_t reps, int32_t* tile, int32_t* per_sm, void* stream);
int gsph_ensemble_launch_count(const gsph_ensemble* e, int64_t* count);
/* text of the last failure on `e` (or of the last failed gsph_ensemble_create when e is NULL) */
const char* gsph_ensemble_last_error(const gsph_ensemble* e);
/* Failure-path test hook (no counterpart in the reference): the next gsph_ensemble_compute_derivatives
 * makes simulation `sim`'s SPH work items wait for one density item more than exists, so their
 * device-side waits run out after options.wait_limit_us; that call returns GSPH_E_TIMEOUT with
 * incomplete results, and the ensemble stays usable (upload a state and call again). One-shot; only
 * the host sets up the failure, no GPU fault is involved. */
int gsph_ensemble_inject_stall(gsph_ensemble* e, int32_t sim);

/* ---------------------------------------------------------------------------------------------
 * measurement hooks (no reference counterpart: the reference has no kernel timers; its console
 * frontend prints wall-clock fps only, src/frontends/consoleFrontend.cpp:43-57)
 * ------------------------------------------------------------------------------------------- */
#define GSPH_KSLOT_DENSITY  0   /* density-sum pair kernel                        */
#define GSPH_KSLOT_VGRAD    1   /* velocity-gradient pair kernel (Balsara on)     */
#define GSPH_KSLOT_PAIRS    2   /* acceleration / fused pair kernel               */
#define GSPH_KSLOT_GRAVITY  3   /* gravity-only pair kernel                       */
#define GSPH_KSLOT_STEP     4   /* one whole step (derivatives + integrate)       */
#define GSPH_KSLOT_INTEGRATE 5  /* the leapfrog kernels of integrate              */
#define GSPH_KSLOTS         6
typedef struct gsph_profile {
    double  ms[GSPH_KSLOTS];        /* accumulated device time per slot (CUDA events) */
    int64_t launches[GSPH_KSLOTS];  /* launches timed per slot                         */
} gsph_profile;
/* Turn per-kernel event timing on or off. When on, each pair kernel launch (including those
 * inside the step graph, captured after this call) is bracketed by CUDA events on its stream.
 * Enabling or disabling drops a previously captured step graph. */
int gsph_profile_enable(gsph_ctx* ctx, int on);
/* Wait for the events recorded since the last collect and add their durations to the totals. */
int gsph_profile_collect(gsph_ctx* ctx);
int gsph_profile_read(gsph_ctx* ctx, gsph_profile* out);
int gsph_profile_reset(gsph_ctx* ctx);

/* Softened all-pairs gravitational accelerations that allocate nothing (no counterpart in the
 * reference, whose hot path always runs on buffers it allocated itself).
 * For callers that may not allocate device memory: a host program that hands out all device memory
 * from a pool fixed at start-up, where a library allocating on its own breaks the budget, or a loop
 * that must never stall, since cudaMalloc / cudaFree can synchronise the whole device.
 *   posm: device array of n float4 (x, y, z, m), 16-byte aligned (input)
 *   acc:  device array of n float4, written as (ax, ay, az, 0) (output)
 *   a_i = -G sum_{j != i} m_j r_ij / (r_ij^2 + eps^2)^(3/2), plain FP32, as the gravity pass of
 *   gsph_compute_derivatives.
 * The scratch (padded j-records and partial sums) is one 16 MiB file-scope device array that every
 * GPU loading the library holds until exit; hence n <= 524288, larger n is rejected with
 * GSPH_E_INVALID and a message in gsph_last_error(NULL). The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress); make that first call before any stream capture.
 * Every call on a device shares the array and leaves the last call's data in it: calls whose
 * kernels may overlap on the GPU (different streams without ordering) race. Asynchronous on `stream`.
 * Outside stream capture every call looks the address up again (a device reset moves the array).
 * Failure: if a bounded device-side wait of the gravity kernel gave up (2 s), part of the sum is
 * missing; the call then writes NaN into every component of acc instead of a partial result, and
 * gsph_gravity_accel_static_status reports GSPH_E_TIMEOUT. */
int gsph_gravity_accel_static(const void* posm, int64_t n, double G, double eps, void* acc, void* stream);
/* Status of the last gsph_gravity_accel_static call on the current device: synchronises `stream`
 * and returns GSPH_OK, or GSPH_E_TIMEOUT when a device-side wait of that call gave up (allocates
 * nothing). */
int gsph_gravity_accel_static_status(void* stream);
/* Failure-path test hook: with on != 0, the next gsph_gravity_accel_static call starts with the
 * timeout bit already set in its status word, as if a device-side wait had given up (no wait is
 * made to run out). One-shot. */
int gsph_inject_static_timeout(int on);

/* FP32 FFMA throughput of the current device, measured by a dependent-chain-free FMA kernel
 * running for about `seconds` (the roofline denominator of the FP32-bound pair kernels).
 * Reports TFLOP/s counting an FMA as 2 flops. */
int gsph_measure_fp32_peak(double seconds, double* tflops);

#ifdef __cplusplus
}
#endif
#endif /* GRASPH2_B200_H */
