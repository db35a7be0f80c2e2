// Minimal stand-in declarations so the reference's CUDA sources compile
// without the cuStateVec SDK (which is not installed in this image).
// TEST INFRASTRUCTURE ONLY: used solely to rebuild the reference as a parity
// checker under oracle/_ref/.  Every entry point returns
// CUSTATEVEC_STATUS_NOT_SUPPORTED, so the reference's inverse_walk_cuQuantum
// strategy raises at run time; its structured_adjoint path never calls these.
#pragma once
#include <cstddef>
#include <cstdint>
#include <library_types.h>

typedef struct custatevecContext *custatevecHandle_t;

typedef enum {
  CUSTATEVEC_STATUS_SUCCESS = 0,
  CUSTATEVEC_STATUS_NOT_SUPPORTED = 15
} custatevecStatus_t;

typedef enum {
  CUSTATEVEC_PAULI_I = 0,
  CUSTATEVEC_PAULI_X = 1,
  CUSTATEVEC_PAULI_Y = 2,
  CUSTATEVEC_PAULI_Z = 3
} custatevecPauli_t;

typedef enum { CUSTATEVEC_MATRIX_LAYOUT_COL = 0, CUSTATEVEC_MATRIX_LAYOUT_ROW = 1 } custatevecMatrixLayout_t;

typedef enum { CUSTATEVEC_COMPUTE_DEFAULT = 0, CUSTATEVEC_COMPUTE_64F = 16 } custatevecComputeType_t;

extern "C" {
custatevecStatus_t custatevecCreate(custatevecHandle_t *handle);
custatevecStatus_t custatevecDestroy(custatevecHandle_t handle);
const char *custatevecGetErrorName(custatevecStatus_t status);
const char *custatevecGetErrorString(custatevecStatus_t status);
custatevecStatus_t custatevecApplyPauliRotation(
    custatevecHandle_t handle, void *sv, cudaDataType_t svDataType, uint32_t nIndexBits,
    double theta, const custatevecPauli_t *paulis, const int32_t *targets, uint32_t nTargets,
    const int32_t *controls, const int32_t *controlBitValues, uint32_t nControls);
custatevecStatus_t custatevecApplyMatrixGetWorkspaceSize(
    custatevecHandle_t handle, cudaDataType_t svDataType, uint32_t nIndexBits,
    const void *matrix, cudaDataType_t matrixDataType, custatevecMatrixLayout_t layout,
    int32_t adjoint, uint32_t nTargets, uint32_t nControls,
    custatevecComputeType_t computeType, size_t *extraWorkspaceSizeInBytes);
custatevecStatus_t custatevecApplyMatrix(
    custatevecHandle_t handle, void *sv, cudaDataType_t svDataType, uint32_t nIndexBits,
    const void *matrix, cudaDataType_t matrixDataType, custatevecMatrixLayout_t layout,
    int32_t adjoint, const int32_t *targets, uint32_t nTargets, const int32_t *controls,
    const int32_t *controlBitValues, uint32_t nControls, custatevecComputeType_t computeType,
    void *extraWorkspace, size_t extraWorkspaceSizeInBytes);
}
