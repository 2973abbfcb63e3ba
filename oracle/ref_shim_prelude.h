/* Force-included into every reference translation unit by oracle/Makefile.
 * The reference predates C++11 headers hygiene: it relies on transitive
 * includes of <cstdlib>/<cmath>/<cstdio>/<cstring>, and calls abs() on an
 * unsigned int in include/delfem/elem_ary.h:88, which g++ 13 rejects as
 * ambiguous.  The overload below is the identity, which is what abs() of an
 * unsigned value means. */
#ifndef DFM_REF_SHIM_PRELUDE_H
#define DFM_REF_SHIM_PRELUDE_H
#ifdef __cplusplus
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
inline unsigned int abs(unsigned int x) { return x; }
#endif
#endif
