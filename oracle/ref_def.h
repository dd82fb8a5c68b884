/* oracle/ref_def.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Force-included (g++ -include) ahead of every reference source file that
 * oracle/Makefile compiles from its place in the reference tree. It defines the
 * include guard of the reference's src/def.h (def.h:23-24), so that file's own
 * body is skipped, and supplies the same macro names (def.h:29-76).
 *
 * The compile-time parameters that the benchmark configurations change
 * (TIME_STEP, nBubbles, Trad, DeltaR, TEST, expansion, ALPHAVAL, Mpl,
 * memorysave, WallTracking) become run-time globals, so one build of the
 * reference serves every configuration. Every use of these macros in the
 * reference is an expression context (e.g. bubble.cpp:276, 870; main.cpp:175),
 * so a variable in place of a literal changes no arithmetic. Output-only
 * switches are fixed to "no plots, no videos". The defaults below equal
 * def.h's values.
 */
#ifndef CB_REF_DEF_H
#define CB_REF_DEF_H
#define DEF_H 1

extern double cbref_time_step;   /* def.h:33  TIME_STEP 0.004 */
extern int cbref_nbubbles;       /* def.h:46  nBubbles 5 */
extern double cbref_trad;        /* def.h:48  Trad 0.2 */
extern double cbref_deltar;      /* def.h:50  DeltaR 0. */
extern int cbref_test;           /* def.h:51  TEST 0 */
extern int cbref_expansion;      /* def.h:56  expansion 0 */
extern int cbref_alpha;          /* def.h:57  ALPHAVAL 0 */
extern double cbref_mpl;         /* def.h:58  Mpl 200.0 */
extern int cbref_memorysave;     /* def.h:64  memorysave 0 */
extern int cbref_walltracking;   /* def.h:72  WallTracking 0 */

#define D_default 2
#define nGrids_default 512
#define L_default 32
#define nt_default 1000
#define TIME_STEP (cbref_time_step)

#define c_default 4.
#define readxns_default 1
#define nBubbles (cbref_nbubbles)
#define fixedseed 1
#define Trad (cbref_trad)
#define DeltaR (cbref_deltar)
#define TEST (cbref_test)

#define expansion (cbref_expansion)
#define ALPHAVAL (cbref_alpha)
#define Mpl (cbref_mpl)

#define Path_default "./"
#define memorysave (cbref_memorysave)
#define OutEnergyEvery 40
#define nSnapshots 20
#define SnapshotSpacing 0
#define FFT 1
#define Full1DFieldEvery 100
#define WallTracking (cbref_walltracking)
#define WallTrackEvery 400
#define plotsnapshots 0
#define makevideos 0

#endif
