/* The reference declares no 2P force expansion (SE_fgg.h:24-27), so its
 * SE_FGG_expand_all_SSE_force does not resolve in a -DTWO_PERIODIC build.
 * This stub lets that build load; calling the 2P force expansion aborts. */
#include <stdlib.h>
int __FGG_EXPA_FORCE(void) { abort(); return 0; }
