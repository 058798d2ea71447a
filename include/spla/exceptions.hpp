/* Exception hierarchy of the C++ interface; each maps to one SplaError code.
 * Class names and codes equal the reference's (include/spla/exceptions.hpp:41-172). */
#ifndef SPLA_EXCEPTIONS_HPP
#define SPLA_EXCEPTIONS_HPP
#include <stdexcept>
#include "spla/config.h"
#include "spla/errors.h"

namespace spla {

class SPLA_EXPORT GenericError : public std::exception {
public:
  const char* what() const noexcept override { return "SPLA: Generic error"; }
  virtual SplaError error_code() const noexcept { return SPLA_UNKNOWN_ERROR; }
};

#define SPLA_B200_DECLARE_ERROR(Name, Base, Code, Text)                        \
  class SPLA_EXPORT Name : public Base {                                       \
  public:                                                                      \
    const char* what() const noexcept override { return Text; }               \
    SplaError error_code() const noexcept override { return Code; }           \
  };

SPLA_B200_DECLARE_ERROR(InternalError, GenericError, SPLA_INTERNAL_ERROR, "SPLA: Internal error")
SPLA_B200_DECLARE_ERROR(InvalidParameterError, GenericError, SPLA_INVALID_PARAMETER_ERROR,
                        "SPLA: Invalid parameter error")
SPLA_B200_DECLARE_ERROR(InvalidPointerError, GenericError, SPLA_INVALID_POINTER_ERROR,
                        "SPLA: Invalid pointer error")
SPLA_B200_DECLARE_ERROR(InvalidAllocatorFunctionError, GenericError,
                        SPLA_INVALID_ALLOCATOR_FUNCTION, "SPLA: Invalid allocator function error")
SPLA_B200_DECLARE_ERROR(MPIError, GenericError, SPLA_MPI_ERROR, "SPLA: MPI error")
SPLA_B200_DECLARE_ERROR(MPIAllocError, MPIError, SPLA_MPI_ALLOCATION_ERROR,
                        "SPLA: MPI memory allocation error")
SPLA_B200_DECLARE_ERROR(MPIThreadSupportError, MPIError, SPLA_MPI_THREAD_SUPPORT_ERROR,
                        "SPLA: MPI multi-threading support not sufficient")
SPLA_B200_DECLARE_ERROR(GPUError, GenericError, SPLA_GPU_ERROR, "SPLA: GPU error")
SPLA_B200_DECLARE_ERROR(GPUSupportError, GPUError, SPLA_GPU_SUPPORT_ERROR,
                        "SPLA: Not compiled with GPU support")
SPLA_B200_DECLARE_ERROR(GPUAllocationError, GPUError, SPLA_GPU_ALLOCATION_ERROR,
                        "SPLA: GPU allocation error")
SPLA_B200_DECLARE_ERROR(GPULaunchError, GPUError, SPLA_GPU_LAUNCH_ERROR, "SPLA: GPU launch error")
SPLA_B200_DECLARE_ERROR(GPUNoDeviceError, GPUError, SPLA_GPU_NO_DEVICE_ERROR,
                        "SPLA: GPU no device error")
SPLA_B200_DECLARE_ERROR(GPUInvalidValueError, GPUError, SPLA_GPU_INVALID_VALUE_ERROR,
                        "SPLA: GPU invalid value error")
SPLA_B200_DECLARE_ERROR(GPUInvalidDevicePointerError, GPUError,
                        SPLA_GPU_INVALID_DEVICE_POINTER_ERROR,
                        "SPLA: GPU invalid device pointer error")
SPLA_B200_DECLARE_ERROR(GPUBlasError, GPUError, SPLA_GPU_BLAS_ERROR, "SPLA: GPU BLAS error")

#undef SPLA_B200_DECLARE_ERROR
}  // namespace spla
#endif
