/*
 * CL/cl.h -- minimal stand-in for the OpenCL header, written for this project.
 *
 * TEST INFRASTRUCTURE ONLY. It exists so that the reference's own
 * gpair1/trunk/gpair.c (whose gpu.h includes <CL/cl.h>) compiles unchanged
 * into the oracle library oracle/_ref/libgpair_ref_main.so, which the tests
 * use to call the reference's init_data (gpair1/trunk/gpair.c:997-1066).
 * No OpenCL runtime exists here and nothing in that library calls one.
 *
 * Only the type names gpu.h and gpair.c use are declared, as opaque handles
 * and as vector structs with the .s0 .. .s3 components that gpair.c writes.
 */
#ifndef GPAIR_ORACLE_CL_SHIM_H
#define GPAIR_ORACLE_CL_SHIM_H

#include <stdint.h>

typedef int32_t cl_int;
typedef uint32_t cl_uint;
typedef struct oracle_cl_mem_ *cl_mem;
typedef struct oracle_cl_program_ *cl_program;
typedef struct oracle_cl_kernel_ *cl_kernel;
typedef struct oracle_cl_device_ *cl_device_id;

typedef struct { float s0, s1; } cl_float2;
typedef struct { float s0, s1, s2, s3; } cl_float4;
typedef struct { int64_t s0, s1, s2, s3; } cl_long4;
typedef struct { int16_t s0, s1, s2, s3; } cl_short4;

#endif
