/*
 * cl_compat.h — the few OpenCL type names that clSpMV's public headers use
 * in their signatures (cl_device_type, cl_context, cl_command_queue,
 * cl_mem), so that callers written against those headers compile and link
 * against libclspmv_b200 without an OpenCL installation.
 *
 * The struct tags are OpenCL's own, so the types are identical when
 * CL/cl.h is included first. In this library a cl_mem is a CUDA device
 * pointer to float, a cl_command_queue is a cudaStream_t (NULL: the legacy
 * default stream) and a cl_context is unused; cl_device_type is ignored
 * (the current CUDA device runs everything).
 */
#ifndef CLSPMV_CL_COMPAT_H
#define CLSPMV_CL_COMPAT_H

#include <stdint.h>

#ifndef __OPENCL_CL_H
typedef uint64_t cl_device_type;
typedef struct _cl_context* cl_context;
typedef struct _cl_command_queue* cl_command_queue;
typedef struct _cl_mem* cl_mem;
#ifndef CL_DEVICE_TYPE_DEFAULT
#define CL_DEVICE_TYPE_DEFAULT (1 << 0)
#define CL_DEVICE_TYPE_CPU (1 << 1)
#define CL_DEVICE_TYPE_GPU (1 << 2)
#define CL_DEVICE_TYPE_ACCELERATOR (1 << 3)
#endif
#endif

#endif /* CLSPMV_CL_COMPAT_H */
