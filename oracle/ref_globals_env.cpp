/* oracle/ref_globals_env.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Definitions of the def.h parameters that oracle/ref_def.h turned into
 * variables, for the reference's own executable (src/main.cpp built in
 * place). Each starts at def.h's value and can be changed through an
 * environment variable, so the unmodified main.cpp can run any benchmark
 * configuration: CBREF_DT, CBREF_NBUBBLES, CBREF_TRAD, CBREF_DELTAR,
 * CBREF_TEST, CBREF_EXPANSION, CBREF_ALPHA, CBREF_MPL, CBREF_MEMORYSAVE,
 * CBREF_WALLTRACKING. */
#include <cstdlib>

static double envd(const char *k, double v) { const char *s = std::getenv(k); return s ? std::atof(s) : v; }
static int envi(const char *k, int v) { const char *s = std::getenv(k); return s ? std::atoi(s) : v; }

double cbref_time_step = envd("CBREF_DT", 0.004);
int cbref_nbubbles = envi("CBREF_NBUBBLES", 5);
double cbref_trad = envd("CBREF_TRAD", 0.2);
double cbref_deltar = envd("CBREF_DELTAR", 0.0);
int cbref_test = envi("CBREF_TEST", 0);
int cbref_expansion = envi("CBREF_EXPANSION", 0);
int cbref_alpha = envi("CBREF_ALPHA", 0);
double cbref_mpl = envd("CBREF_MPL", 200.0);
int cbref_memorysave = envi("CBREF_MEMORYSAVE", 0);
int cbref_walltracking = envi("CBREF_WALLTRACKING", 0);
