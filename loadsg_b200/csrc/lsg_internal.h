// Library-internal interface between the operator (lsg_device.cu) and the
// batched solver (lsg_batch.cu).  Not part of the C-ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>

#include "lsg_plan.h"

struct lsg_operator;

namespace lsg_internal {

// Uploads a (possibly concatenated) plan; every part needs its coefficient.
int create_from_plan(lsg::Plan&& plan, lsg_operator** out);
int set_part_coefficient(lsg_operator* op, int part, int32_t family, const double* params, int32_t nparams);
// y = A x on the active entries of every part (inactive entries untouched)
int matvec64(lsg_operator* op, const double* x, double* y, cudaStream_t st);
int matvec32(lsg_operator* op, const float* x, float* y, cudaStream_t st);
// work buffers and kernel attributes (call before a stream capture)
int prepare_precision(lsg_operator* op, bool fp32);
const uint8_t* active(lsg_operator* op);
// exact Jacobi diagonal, computed once per coefficient
int jacobi_diag(lsg_operator* op, cudaStream_t st, const double** diag);
bool has_coefficient(const lsg_operator* op);
const lsg::Plan& plan(const lsg_operator* op);
size_t device_bytes(const lsg_operator* op);
int64_t matvec_launch_count(const lsg_operator* op, bool f32);
int fail_msg(int code, const char* msg);
int autotune(lsg_operator* op, int32_t precision, int32_t reps);
// y = A x with coefficient 1 in form 0 (stiffness) or 1 (mass), FP64
int matvec64_unit(lsg_operator* op, int form, const double* x, double* y, cudaStream_t st);
// per-operator state of the basis transforms (lsg_basis.cu)
std::shared_ptr<void>& basis_slot(lsg_operator* op);
// calcPrewByNodal on device vectors (lsg_basis.cu)
int prew_by_nodal_dev(lsg_operator* op, double* prew, const double* u, cudaStream_t st);
// per-operator tables of the boundary-data right-hand sides (lsg_bdrhs.cu)
std::shared_ptr<void>& bdrhs_slot(lsg_operator* op);

}  // namespace lsg_internal
