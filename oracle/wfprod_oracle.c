/* Wave-function product oracle: filled in with the MT / PW restatements. */
#include <stdint.h>
int oracle_wfprod_version(void) { return 1; }
