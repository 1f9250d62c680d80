// ORACLE — test infrastructure only (see oracle/oracle.c).
//
// C-linkage entry points over the reference's own host routines, compiled
// unmodified from LINPACK/src/host/linpack_data.cpp (gefa_ref_nopvt :166-196,
// gesl_ref_nopvt :199-229, gefa_ref :72-119, gesl_ref :121-156) by
// oracle/Makefile into oracle/_ref/.  REF_SUFFIX is _f32 or _f64 depending on
// HOST_DATA_TYPE (oracle/refstub/parameters.h).
#include "linpack_data.hpp"

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define REF(name) CAT(ref_##name, REF_SUFFIX)

extern "C" {
void REF(gefa_nopvt)(HOST_DATA_TYPE* a, unsigned n, unsigned lda) { linpack::gefa_ref_nopvt(a, n, lda); }
void REF(gesl_nopvt)(HOST_DATA_TYPE* a, HOST_DATA_TYPE* b, unsigned n, unsigned lda) {
    linpack::gesl_ref_nopvt(a, b, n, lda);
}
void REF(gefa_pvt)(HOST_DATA_TYPE* a, unsigned n, unsigned lda, int* ipvt) {
    linpack::gefa_ref(a, n, lda, ipvt);
}
void REF(gesl_pvt)(HOST_DATA_TYPE* a, HOST_DATA_TYPE* b, int* ipvt, unsigned n, unsigned lda) {
    linpack::gesl_ref(a, b, ipvt, n, lda);
}
}
