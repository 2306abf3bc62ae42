/* Minimal stand-in for the OpenCL 1.2 host API header, written for this
 * project: types, the constants the reference's sources name (distinct values,
 * not the Khronos ones) and the entry points they call. Implemented by
 * oracle/ref_codegen/stubs.cpp, which runs no device code: it exists so that the
 * reference's own DAG, fusion and kernel generators can run on the CPU and
 * print the OpenCL kernels they generate. TEST INFRASTRUCTURE ONLY. */
#ifndef MAP_STUB_CL_H
#define MAP_STUB_CL_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef int32_t cl_int;
typedef uint32_t cl_uint;
typedef uint64_t cl_ulong;
typedef cl_uint cl_bool;
typedef cl_ulong cl_bitfield;
typedef cl_bitfield cl_device_type;
typedef cl_uint cl_platform_info;
typedef cl_uint cl_device_info;
typedef cl_bitfield cl_mem_flags;
typedef cl_bitfield cl_map_flags;
typedef cl_bitfield cl_command_queue_properties;
typedef intptr_t cl_context_properties;
typedef intptr_t cl_device_partition_property;
typedef cl_uint cl_program_build_info;
typedef cl_int cl_build_status;
typedef cl_uint cl_buffer_create_type;
typedef struct _cl_platform_id *cl_platform_id;
typedef struct _cl_device_id *cl_device_id;
typedef struct _cl_context *cl_context;
typedef struct _cl_command_queue *cl_command_queue;
typedef struct _cl_mem *cl_mem;
typedef struct _cl_program *cl_program;
typedef struct _cl_kernel *cl_kernel;
typedef struct _cl_event *cl_event;
typedef struct _cl_buffer_region { size_t origin; size_t size; } cl_buffer_region;

#define CL_SUCCESS 0
#define CL_FALSE 0
#define CL_TRUE 1
#define CL_BUILD_PROGRAM_FAILURE (-1)
#define CL_COMPILER_NOT_AVAILABLE (-2)
#define CL_COMPILE_PROGRAM_FAILURE (-3)
#define CL_D3D10_RESOURCE_ALREADY_ACQUIRED_KHR (-4)
#define CL_D3D10_RESOURCE_NOT_ACQUIRED_KHR (-5)
#define CL_DEVICE_NOT_FOUND (-6)
#define CL_DEVICE_PARTITION_FAILED (-7)
#define CL_EXEC_STATUS_ERROR_FOR_EVENTS_IN_WAIT_LIST (-8)
#define CL_IMAGE_FORMAT_MISMATCH (-9)
#define CL_IMAGE_FORMAT_NOT_SUPPORTED (-10)
#define CL_INVALID_ARG_INDEX (-11)
#define CL_INVALID_ARG_SIZE (-12)
#define CL_INVALID_ARG_VALUE (-13)
#define CL_INVALID_BINARY (-14)
#define CL_INVALID_BUFFER_SIZE (-15)
#define CL_INVALID_BUILD_OPTIONS (-16)
#define CL_INVALID_COMMAND_QUEUE (-17)
#define CL_INVALID_COMPILER_OPTIONS (-18)
#define CL_INVALID_CONTEXT (-19)
#define CL_INVALID_D3D10_DEVICE_KHR (-20)
#define CL_INVALID_D3D10_RESOURCE_KHR (-21)
#define CL_INVALID_DEVICE (-22)
#define CL_INVALID_DEVICE_PARTITION_COUNT (-23)
#define CL_INVALID_DEVICE_TYPE (-24)
#define CL_INVALID_EVENT (-25)
#define CL_INVALID_EVENT_WAIT_LIST (-26)
#define CL_INVALID_GLOBAL_OFFSET (-27)
#define CL_INVALID_GLOBAL_WORK_SIZE (-28)
#define CL_INVALID_GL_OBJECT (-29)
#define CL_INVALID_GL_SHAREGROUP_REFERENCE_KHR (-30)
#define CL_INVALID_HOST_PTR (-31)
#define CL_INVALID_IMAGE_DESCRIPTOR (-32)
#define CL_INVALID_IMAGE_FORMAT_DESCRIPTOR (-33)
#define CL_INVALID_IMAGE_SIZE (-34)
#define CL_INVALID_KERNEL (-35)
#define CL_INVALID_KERNEL_ARGS (-36)
#define CL_INVALID_KERNEL_DEFINITION (-37)
#define CL_INVALID_KERNEL_NAME (-38)
#define CL_INVALID_LINKER_OPTIONS (-39)
#define CL_INVALID_MEM_OBJECT (-40)
#define CL_INVALID_MIP_LEVEL (-41)
#define CL_INVALID_OPERATION (-42)
#define CL_INVALID_PLATFORM (-43)
#define CL_INVALID_PROGRAM (-44)
#define CL_INVALID_PROGRAM_EXECUTABLE (-45)
#define CL_INVALID_PROPERTY (-46)
#define CL_INVALID_QUEUE_PROPERTIES (-47)
#define CL_INVALID_SAMPLER (-48)
#define CL_INVALID_VALUE (-49)
#define CL_INVALID_WORK_DIMENSION (-50)
#define CL_INVALID_WORK_GROUP_SIZE (-51)
#define CL_INVALID_WORK_ITEM_SIZE (-52)
#define CL_KERNEL_ARG_INFO_NOT_AVAILABLE (-53)
#define CL_LINKER_NOT_AVAILABLE (-54)
#define CL_LINK_PROGRAM_FAILURE (-55)
#define CL_MAP_FAILURE (-56)
#define CL_MEM_COPY_OVERLAP (-58)
#define CL_MEM_OBJECT_ALLOCATION_FAILURE (-59)
#define CL_MISALIGNED_SUB_BUFFER_OFFSET (-60)
#define CL_OUT_OF_HOST_MEMORY (-61)
#define CL_OUT_OF_RESOURCES (-62)
#define CL_PROFILING_INFO_NOT_AVAILABLE (-63)
#define CL_BUFFER_CREATE_TYPE_REGION 0x2000
#define CL_CONTEXT_PLATFORM 0x2001
#define CL_DEVICE_ADDRESS_BITS 0x2002
#define CL_DEVICE_AVAILABLE 0x2003
#define CL_DEVICE_COMPILER_AVAILABLE 0x2004
#define CL_DEVICE_ENDIAN_LITTLE 0x2005
#define CL_DEVICE_ERROR_CORRECTION_SUPPORT 0x2006
#define CL_DEVICE_EXECUTION_CAPABILITIES 0x2007
#define CL_DEVICE_EXTENSIONS 0x2008
#define CL_DEVICE_GLOBAL_MEM_CACHELINE_SIZE 0x2009
#define CL_DEVICE_GLOBAL_MEM_CACHE_SIZE 0x200a
#define CL_DEVICE_GLOBAL_MEM_CACHE_TYPE 0x200b
#define CL_DEVICE_GLOBAL_MEM_SIZE 0x200c
#define CL_DEVICE_IMAGE2D_MAX_HEIGHT 0x200d
#define CL_DEVICE_IMAGE2D_MAX_WIDTH 0x200e
#define CL_DEVICE_IMAGE3D_MAX_DEPTH 0x200f
#define CL_DEVICE_IMAGE3D_MAX_HEIGHT 0x2010
#define CL_DEVICE_IMAGE3D_MAX_WIDTH 0x2011
#define CL_DEVICE_IMAGE_SUPPORT 0x2012
#define CL_DEVICE_LOCAL_MEM_SIZE 0x2013
#define CL_DEVICE_LOCAL_MEM_TYPE 0x2014
#define CL_DEVICE_MAX_CLOCK_FREQUENCY 0x2015
#define CL_DEVICE_MAX_COMPUTE_UNITS 0x2016
#define CL_DEVICE_MAX_CONSTANT_ARGS 0x2017
#define CL_DEVICE_MAX_CONSTANT_BUFFER_SIZE 0x2018
#define CL_DEVICE_MAX_MEM_ALLOC_SIZE 0x2019
#define CL_DEVICE_MAX_PARAMETER_SIZE 0x201a
#define CL_DEVICE_MAX_READ_IMAGE_ARGS 0x201b
#define CL_DEVICE_MAX_SAMPLERS 0x201c
#define CL_DEVICE_MAX_WORK_GROUP_SIZE 0x201d
#define CL_DEVICE_MAX_WORK_ITEM_DIMENSIONS 0x201e
#define CL_DEVICE_MAX_WORK_ITEM_SIZES 0x201f
#define CL_DEVICE_MAX_WRITE_IMAGE_ARGS 0x2020
#define CL_DEVICE_MEM_BASE_ADDR_ALIGN 0x2021
#define CL_DEVICE_MIN_DATA_TYPE_ALIGN_SIZE 0x2022
#define CL_DEVICE_NAME 0x2023
#define CL_DEVICE_NOT_AVAILABLE 0x2024
#define CL_DEVICE_PARTITION_BY_COUNTS 0x2025
#define CL_DEVICE_PARTITION_BY_COUNTS_LIST_END 0x2026
#define CL_DEVICE_PLATFORM 0x2027
#define CL_DEVICE_PREFERRED_VECTOR_WIDTH_CHAR 0x2028
#define CL_DEVICE_PREFERRED_VECTOR_WIDTH_DOUBLE 0x2029
#define CL_DEVICE_PREFERRED_VECTOR_WIDTH_FLOAT 0x202a
#define CL_DEVICE_PREFERRED_VECTOR_WIDTH_INT 0x202b
#define CL_DEVICE_PREFERRED_VECTOR_WIDTH_LONG 0x202c
#define CL_DEVICE_PREFERRED_VECTOR_WIDTH_SHORT 0x202d
#define CL_DEVICE_PROFILE 0x202e
#define CL_DEVICE_PROFILING_TIMER_RESOLUTION 0x202f
#define CL_DEVICE_QUEUE_PROPERTIES 0x2030
#define CL_DEVICE_SINGLE_FP_CONFIG 0x2031
#define CL_DEVICE_TYPE 0x2032
#define CL_DEVICE_VENDOR 0x2033
#define CL_DEVICE_VENDOR_ID 0x2034
#define CL_DEVICE_VERSION 0x2035
#define CL_PLATFORM_EXTENSIONS 0x2036
#define CL_PLATFORM_NAME 0x2037
#define CL_PLATFORM_PROFILE 0x2038
#define CL_PLATFORM_VENDOR 0x2039
#define CL_PLATFORM_VERSION 0x203a
#define CL_PROGRAM_BUILD_LOG 0x203b
#define CL_PROGRAM_BUILD_STATUS 0x203c
#define CL_DEVICE_TYPE_ACCELERATOR ((cl_bitfield)1 << 0)
#define CL_DEVICE_TYPE_CPU ((cl_bitfield)1 << 1)
#define CL_DEVICE_TYPE_CUSTOM ((cl_bitfield)1 << 2)
#define CL_DEVICE_TYPE_DEFAULT ((cl_bitfield)1 << 3)
#define CL_DEVICE_TYPE_GPU ((cl_bitfield)1 << 4)
#define CL_MAP_READ ((cl_bitfield)1 << 5)
#define CL_MAP_WRITE ((cl_bitfield)1 << 6)
#define CL_MAP_WRITE_INVALIDATE_REGION ((cl_bitfield)1 << 11)
#define CL_MEM_ALLOC_HOST_PTR ((cl_bitfield)1 << 7)
#define CL_MEM_READ_ONLY ((cl_bitfield)1 << 8)
#define CL_MEM_READ_WRITE ((cl_bitfield)1 << 9)
#define CL_MEM_WRITE_ONLY ((cl_bitfield)1 << 10)
#define CL_DEVICE_TYPE_ALL 0xFFFFFFFF

cl_int clGetPlatformIDs(cl_uint, cl_platform_id *, cl_uint *);
cl_int clGetPlatformInfo(cl_platform_id, cl_platform_info, size_t, void *, size_t *);
cl_int clGetDeviceIDs(cl_platform_id, cl_device_type, cl_uint, cl_device_id *, cl_uint *);
cl_int clGetDeviceInfo(cl_device_id, cl_device_info, size_t, void *, size_t *);
cl_int clCreateSubDevices(cl_device_id, const cl_device_partition_property *, cl_uint, cl_device_id *, cl_uint *);
cl_context clCreateContext(const cl_context_properties *, cl_uint, const cl_device_id *,
                           void (*)(const char *, const void *, size_t, void *), void *, cl_int *);
cl_int clReleaseContext(cl_context);
cl_command_queue clCreateCommandQueue(cl_context, cl_device_id, cl_command_queue_properties, cl_int *);
cl_int clReleaseCommandQueue(cl_command_queue);
cl_mem clCreateBuffer(cl_context, cl_mem_flags, size_t, void *, cl_int *);
cl_mem clCreateSubBuffer(cl_mem, cl_mem_flags, cl_buffer_create_type, const void *, cl_int *);
cl_int clReleaseMemObject(cl_mem);
cl_program clCreateProgramWithSource(cl_context, cl_uint, const char **, const size_t *, cl_int *);
cl_int clBuildProgram(cl_program, cl_uint, const cl_device_id *, const char *, void (*)(cl_program, void *), void *);
cl_int clGetProgramBuildInfo(cl_program, cl_device_id, cl_program_build_info, size_t, void *, size_t *);
cl_int clReleaseProgram(cl_program);
cl_kernel clCreateKernel(cl_program, const char *, cl_int *);
cl_int clReleaseKernel(cl_kernel);
cl_int clSetKernelArg(cl_kernel, cl_uint, size_t, const void *);
cl_int clEnqueueNDRangeKernel(cl_command_queue, cl_kernel, cl_uint, const size_t *, const size_t *, const size_t *,
                              cl_uint, const cl_event *, cl_event *);
cl_int clEnqueueReadBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t, void *, cl_uint, const cl_event *, cl_event *);
cl_int clEnqueueWriteBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t, const void *, cl_uint, const cl_event *,
                            cl_event *);
cl_int clEnqueueCopyBuffer(cl_command_queue, cl_mem, cl_mem, size_t, size_t, size_t, cl_uint, const cl_event *, cl_event *);
cl_int clEnqueueFillBuffer(cl_command_queue, cl_mem, const void *, size_t, size_t, size_t, cl_uint, const cl_event *,
                           cl_event *);
void *clEnqueueMapBuffer(cl_command_queue, cl_mem, cl_bool, cl_map_flags, size_t, size_t, cl_uint, const cl_event *,
                         cl_event *, cl_int *);
cl_int clEnqueueUnmapMemObject(cl_command_queue, cl_mem, void *, cl_uint, const cl_event *, cl_event *);
cl_event clCreateUserEvent(cl_context, cl_int *);
cl_int clReleaseEvent(cl_event);
cl_int clFinish(cl_command_queue);
#ifdef __cplusplus
}
#endif
#endif
