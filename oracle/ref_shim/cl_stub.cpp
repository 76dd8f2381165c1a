// Definitions for the OpenCL stub header: every call fails with an error code
// and touches nothing, so the reference's GPU classes link but never run.
// Test infrastructure for the reference CPU oracle build only.
#include "CL/opencl.h"

extern "C" {

cl_int clGetPlatformIDs(cl_uint, cl_platform_id*, cl_uint* n) { if (n) *n = 0; return CL_INVALID_PLATFORM; }
cl_int clGetDeviceIDs(cl_platform_id, cl_device_type, cl_uint, cl_device_id*, cl_uint* n) { if (n) *n = 0; return CL_DEVICE_NOT_FOUND; }
cl_int clGetDeviceInfo(cl_device_id, cl_device_info, size_t, void*, size_t*) { return CL_INVALID_VALUE; }
cl_context clCreateContext(const cl_context_properties*, cl_uint, const cl_device_id*,
                           void (*)(const char*, const void*, size_t, void*), void*, cl_int* e) { if (e) *e = CL_INVALID_PLATFORM; return nullptr; }
cl_command_queue clCreateCommandQueue(cl_context, cl_device_id, cl_command_queue_properties, cl_int* e) { if (e) *e = CL_INVALID_PLATFORM; return nullptr; }
cl_mem clCreateBuffer(cl_context, cl_mem_flags, size_t, void*, cl_int* e) { if (e) *e = CL_INVALID_PLATFORM; return nullptr; }
cl_int clReleaseMemObject(cl_mem) { return CL_INVALID_VALUE; }
cl_int clEnqueueWriteBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t, const void*, cl_uint, const cl_event*, cl_event*) { return CL_INVALID_VALUE; }
cl_int clEnqueueReadBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t, void*, cl_uint, const cl_event*, cl_event*) { return CL_INVALID_VALUE; }
cl_int clEnqueueNDRangeKernel(cl_command_queue, cl_kernel, cl_uint, const size_t*, const size_t*, const size_t*, cl_uint, const cl_event*, cl_event*) { return CL_INVALID_VALUE; }
cl_int clSetKernelArg(cl_kernel, cl_uint, size_t, const void*) { return CL_INVALID_VALUE; }
cl_int clFinish(cl_command_queue) { return CL_SUCCESS; }
cl_int clWaitForEvents(cl_uint, const cl_event*) { return CL_INVALID_VALUE; }
cl_int clReleaseEvent(cl_event) { return CL_INVALID_VALUE; }
cl_program clCreateProgramWithSource(cl_context, cl_uint, const char**, const size_t*, cl_int* e) { if (e) *e = CL_INVALID_VALUE; return nullptr; }
cl_int clBuildProgram(cl_program, cl_uint, const cl_device_id*, const char*, void (*)(cl_program, void*), void*) { return CL_INVALID_VALUE; }
cl_int clGetProgramBuildInfo(cl_program, cl_device_id, cl_program_build_info, size_t, void*, size_t* s) { if (s) *s = 0; return CL_INVALID_VALUE; }
cl_int clCreateKernelsInProgram(cl_program, cl_uint, cl_kernel*, cl_uint* n) { if (n) *n = 0; return CL_INVALID_VALUE; }
cl_kernel clCreateKernel(cl_program, const char*, cl_int* e) { if (e) *e = CL_INVALID_VALUE; return nullptr; }
cl_int clRetainProgram(cl_program) { return CL_INVALID_VALUE; }
cl_int clRetainKernel(cl_kernel) { return CL_INVALID_VALUE; }
cl_int clReleaseProgram(cl_program) { return CL_INVALID_VALUE; }
cl_int clReleaseKernel(cl_kernel) { return CL_INVALID_VALUE; }

}
