/* Force-included (-include) into the reference build by oracle/build_ref.sh.
 * The reference calls memcpy on overlapping ranges (include/graph.h:700,735;
 * include/btree.h:360,368,501), which glibc's optimised memcpy corrupts under
 * -Ofast; memmove is the defined operation for overlapping copies.
 * libstdc++'s <cstring> #undefs memcpy, so it is pulled in first (its include
 * guard then keeps later inclusions from undoing the macro). */
#ifdef __cplusplus
#include <cstring>
#endif
#include <string.h>
#define memcpy memmove
