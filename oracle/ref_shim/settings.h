/*
 * TEST INFRASTRUCTURE ONLY. Stand-in for GraSPH2's settings/settings.h, configured by -D macros
 * from oracle/build_ref.py so one source builds every physics variant the parity tests use. The
 * names are the reference's own (settings/settings.h:26-185) because the reference's job headers
 * read them; each REF_* macro maps to one of its switches or constants.
 */
#ifndef GRASPH2_SETTINGS_H
#define GRASPH2_SETTINGS_H

#include "types.h"
#include <particles/Particles.h>  /* the host or the CUDA stand-in, by include path */

constexpr Dim dimension = Dim::three;

#if REF_GRAVITY
#define ENABLE_SELF_GRAVITY
#endif
#if REF_SPH
#define ENABLE_SPH
#endif
#if REF_INTEGRATE_DENSITY
#define INTEGRATE_DENSITY
#endif
#if REF_DEAL_WITH_NO_PARTNERS
#define DEAL_WITH_NO_PARTNERS
#endif
#if REF_SOLIDS
#define SOLIDS
#endif

/* Host build: the variable-step kernels of src/integration.h:130-217 are called directly by the
 * parity driver; integrate()'s own variable-step branch launches them with <<<>>>, which a host
 * compiler cannot parse, so the fixed-step branch is the one compiled. CUDA build: integrate()
 * dispatches as the reference does. */
#if defined(__CUDACC__) && REF_VARIABLE_TIMESTEP
#define VARIABLE_TIMESTEP_LEAPFROG
#else
#define FIXED_TIMESTEP_LEAPFROG
#endif
constexpr f1_t fixed_timestep = REF_FIXED_DT;
constexpr f1_t initial_timestep = REF_INITIAL_DT;
constexpr f1_t min_timestep = REF_MIN_DT;
constexpr f1_t max_timestep = REF_MAX_DT;
#if REF_ACCELERATION_CRITERION
#define ACCELERATION_CRITERION
#endif
constexpr f1_t accel_accuracy = REF_ACCEL_ACCURACY;
#if REF_VELOCITY_CRITERION
#define VELOCITY_CRITERION
#endif
constexpr f1_t velocity_accuracy = REF_VELOCITY_ACCURACY;

constexpr f1_t H = REF_H;

constexpr f1_t rho0 = REF_RHO0;
constexpr f1_t BULK = REF_BULK;
constexpr f1_t dBULKdP = REF_DBULKDP;
constexpr f1_t SOUNDSPEED = REF_SOUNDSPEED;
constexpr f1_t shear = REF_SHEAR;

#if REF_PLASTICITY_MIESE
#define PLASTICITY_MIESE
#endif
constexpr f1_t Y = REF_Y;
#if REF_PLASTICITY_MC
#define PLASTICITY_MC
#endif
constexpr f1_t tanfr = REF_TANFR;
constexpr f1_t cohesion = REF_COHESION;

#if REF_CLOHESSY_WILTSHIRE
#define CLOHESSY_WILTSHIRE
#endif
constexpr f1_t cw_n = REF_CW_N;
#if REF_CONSTANT_ACCELERATION
#define CONSTANT_ACCELERATION
#endif
constexpr f3_t constant_acceleration = {REF_CONST_ACC_X, REF_CONST_ACC_Y, REF_CONST_ACC_Z};
#if REF_SIMPLE_BOX_BOUNDARY
#define SIMPLE_BOX_BOUNDARY
#endif
constexpr f3_t simple_box_bound_min = {REF_BOX_MIN, REF_BOX_MIN, REF_BOX_MIN};
constexpr f3_t simple_box_bound_max = {REF_BOX_MAX, REF_BOX_MAX, REF_BOX_MAX};
constexpr f1_t simple_box_bound_reflectiveness = REF_BOX_REFLECT;

#if REF_ARTIFICIAL_VISCOSITY
#define ARTIFICIAL_VISCOSITY
#endif
constexpr f1_t alpha = REF_ALPHA;
#if REF_BALSARA_SWITCH
#define BALSARA_SWITCH
#endif
#if REF_ARTIFICIAL_STRESS
#define ARTIFICIAL_STRESS
#endif
constexpr f1_t mateps = REF_MATEPS;
constexpr f1_t matexp = REF_MATEXP;
constexpr f1_t normalsep = H * REF_NORMALSEP_FRAC;
#if REF_XSPH
#define XSPH
#endif
constexpr f1_t xsph_factor = REF_XSPH_FACTOR;

constexpr size_t BLOCK_SIZE = 256;
constexpr size_t INTEG_BS = BLOCK_SIZE;
constexpr size_t INTEG_PPT = 1;

#endif
