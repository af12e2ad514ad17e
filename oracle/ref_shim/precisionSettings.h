/* TEST INFRASTRUCTURE ONLY. Precision switch of settings/precisionSettings.h:16-17, chosen by the
 * build recipe (oracle/build_ref.py) with -DREF_DOUBLE for the FP64 variant. */
#ifndef GRASPH2_PRECISIONSETTINGS_H
#define GRASPH2_PRECISIONSETTINGS_H
#if defined(REF_DOUBLE)
#define DOUBLE_PRECISION
#else
#define SINGLE_PRECISION
#endif
#endif
