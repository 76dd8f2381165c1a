/*
 * Minimal OpenCL type/API declaration stub used ONLY to compile the reference
 * Aster CPU sources as a test oracle on machines without OpenCL headers.
 * Written from scratch: it declares just the types, constants and entry points
 * that the reference sources name. Every function is defined in cl_stub.cpp and
 * returns an error, so no GPU path of the reference can run through it.
 *
 * Test infrastructure: nothing in the product links this.
 */
#ifndef ASTER_ORACLE_CL_STUB_H
#define ASTER_ORACLE_CL_STUB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t  cl_int;
typedef uint32_t cl_uint;
typedef uint64_t cl_ulong;
typedef uint32_t cl_bool;
typedef cl_ulong cl_bitfield;
typedef cl_bitfield cl_device_type;
typedef cl_bitfield cl_mem_flags;
typedef cl_bitfield cl_command_queue_properties;
typedef cl_bitfield cl_device_fp_config;
typedef cl_uint cl_device_info;
typedef cl_uint cl_program_build_info;
typedef intptr_t cl_context_properties;

typedef union { cl_uint s[2]; struct { cl_uint x, y; }; } cl_uint2;

typedef struct _cl_platform_id*   cl_platform_id;
typedef struct _cl_device_id*     cl_device_id;
typedef struct _cl_context*       cl_context;
typedef struct _cl_command_queue* cl_command_queue;
typedef struct _cl_mem*           cl_mem;
typedef struct _cl_program*       cl_program;
typedef struct _cl_kernel*        cl_kernel;
typedef struct _cl_event*         cl_event;

#define CL_SUCCESS 0
#define CL_DEVICE_NOT_FOUND (-1)
#define CL_INVALID_VALUE (-30)
#define CL_INVALID_PLATFORM (-32)
#define CL_FALSE 0u
#define CL_TRUE 1u
#define CL_DEVICE_TYPE_ALL 0xFFFFFFFFull
#define CL_MEM_READ_WRITE (1ull << 0)
#define CL_MEM_WRITE_ONLY (1ull << 1)
#define CL_MEM_READ_ONLY  (1ull << 2)
#define CL_DEVICE_MAX_COMPUTE_UNITS 0x1002u
#define CL_DEVICE_MAX_CLOCK_FREQUENCY 0x100Cu
#define CL_DEVICE_GLOBAL_MEM_SIZE 0x101Fu
#define CL_DEVICE_DOUBLE_FP_CONFIG 0x1032u
#define CL_PROGRAM_BUILD_LOG 0x1183u

cl_int clGetPlatformIDs(cl_uint, cl_platform_id*, cl_uint*);
cl_int clGetDeviceIDs(cl_platform_id, cl_device_type, cl_uint, cl_device_id*, cl_uint*);
cl_int clGetDeviceInfo(cl_device_id, cl_device_info, size_t, void*, size_t*);
cl_context clCreateContext(const cl_context_properties*, cl_uint, const cl_device_id*,
                           void (*)(const char*, const void*, size_t, void*), void*, cl_int*);
cl_command_queue clCreateCommandQueue(cl_context, cl_device_id, cl_command_queue_properties, cl_int*);
cl_mem clCreateBuffer(cl_context, cl_mem_flags, size_t, void*, cl_int*);
cl_int clReleaseMemObject(cl_mem);
cl_int clEnqueueWriteBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t, const void*,
                            cl_uint, const cl_event*, cl_event*);
cl_int clEnqueueReadBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t, void*,
                           cl_uint, const cl_event*, cl_event*);
cl_int clEnqueueNDRangeKernel(cl_command_queue, cl_kernel, cl_uint, const size_t*, const size_t*,
                              const size_t*, cl_uint, const cl_event*, cl_event*);
cl_int clSetKernelArg(cl_kernel, cl_uint, size_t, const void*);
cl_int clFinish(cl_command_queue);
cl_int clWaitForEvents(cl_uint, const cl_event*);
cl_int clReleaseEvent(cl_event);
cl_program clCreateProgramWithSource(cl_context, cl_uint, const char**, const size_t*, cl_int*);
cl_int clBuildProgram(cl_program, cl_uint, const cl_device_id*, const char*,
                      void (*)(cl_program, void*), void*);
cl_int clGetProgramBuildInfo(cl_program, cl_device_id, cl_program_build_info, size_t, void*, size_t*);
cl_int clCreateKernelsInProgram(cl_program, cl_uint, cl_kernel*, cl_uint*);
cl_kernel clCreateKernel(cl_program, const char*, cl_int*);
cl_int clRetainProgram(cl_program);
cl_int clRetainKernel(cl_kernel);
cl_int clReleaseProgram(cl_program);
cl_int clReleaseKernel(cl_kernel);

#ifdef __cplusplus
}
#endif

#endif
