// Stub definitions for oracle/ref_stub/custatevec.h (see that header).
#include "custatevec.h"

extern "C" {
custatevecStatus_t custatevecCreate(custatevecHandle_t *handle) {
  if (handle) *handle = nullptr;
  return CUSTATEVEC_STATUS_NOT_SUPPORTED;
}
custatevecStatus_t custatevecDestroy(custatevecHandle_t) { return CUSTATEVEC_STATUS_SUCCESS; }
const char *custatevecGetErrorName(custatevecStatus_t s) {
  return s == CUSTATEVEC_STATUS_SUCCESS ? "CUSTATEVEC_STATUS_SUCCESS"
                                        : "CUSTATEVEC_STATUS_NOT_SUPPORTED";
}
const char *custatevecGetErrorString(custatevecStatus_t) {
  return "cuStateVec is not available in this rebuild of the reference";
}
custatevecStatus_t custatevecApplyPauliRotation(custatevecHandle_t, void *, cudaDataType_t,
                                                uint32_t, double, const custatevecPauli_t *,
                                                const int32_t *, uint32_t, const int32_t *,
                                                const int32_t *, uint32_t) {
  return CUSTATEVEC_STATUS_NOT_SUPPORTED;
}
custatevecStatus_t custatevecApplyMatrixGetWorkspaceSize(custatevecHandle_t, cudaDataType_t,
                                                         uint32_t, const void *, cudaDataType_t,
                                                         custatevecMatrixLayout_t, int32_t,
                                                         uint32_t, uint32_t,
                                                         custatevecComputeType_t, size_t *) {
  return CUSTATEVEC_STATUS_NOT_SUPPORTED;
}
custatevecStatus_t custatevecApplyMatrix(custatevecHandle_t, void *, cudaDataType_t, uint32_t,
                                         const void *, cudaDataType_t, custatevecMatrixLayout_t,
                                         int32_t, const int32_t *, uint32_t, const int32_t *,
                                         const int32_t *, uint32_t, custatevecComputeType_t,
                                         void *, size_t) {
  return CUSTATEVEC_STATUS_NOT_SUPPORTED;
}
}
