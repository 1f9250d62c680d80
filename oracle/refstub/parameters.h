// Test infrastructure only (oracle build). Stand-in for the CMake-generated
// LINPACK/src/common/parameters.h.in: HOST_DATA_TYPE is chosen on the compiler
// command line (-DREF_FP64 selects double, the reference's _DP build).
#ifndef ORACLE_REFSTUB_PARAMETERS_H
#define ORACLE_REFSTUB_PARAMETERS_H
#ifdef REF_FP64
#define HOST_DATA_TYPE double
#define DEVICE_DATA_TYPE double
#define _DP
#else
#define HOST_DATA_TYPE float
#define DEVICE_DATA_TYPE float
#endif
#define VERSION "2.6"
#define LOCAL_MEM_BLOCK_LOG 5
#define REGISTER_BLOCK_LOG 3
#define REGISTER_BLOCK_MM_LOG 3
#define DEFAULT_MATRIX_SIZE 2
#define DEFAULT_P_VALUE 1
#endif
