// field_ops.cu -- the reference's optimised pointwise field hooks on the GPU.
//
// Block/FieldOperator.h:149-227 declares, under CUBISM_OPTIMIZED_FIELD_OP,
//   void field{Add,Sub,Mul,Div}2_{double,float}(const T*, const T*, T*, size_t)
//   void field{Add,Sub,Mul,Div}1_{double,float}(const T*, const T,  T*, size_t)
//   void fieldRcp_{double,float}(const T*, const T, T*, size_t)
// and never defines them.  This file defines them with exactly those names so
// a reference build with that option links against this library: dst[i] =
// src0[i] OP src1[i] (or OP scalar), and Rcp dst[i] = src1 * (1 / src0[i])
// (FieldOperator.h:16-30).  Device (and managed) pointers are processed in
// place; host pointers are staged through device memory.  The hooks return
// after the result is in dst.
#include "cn_internal.h"

namespace cn {

enum FieldOpKind { kAdd = 0, kSub = 1, kMul = 2, kDiv = 3, kRcp = 4 };

template <typename T, int OP, bool SCALAR>
__global__ void __launch_bounds__(256)
    field_op_kernel(const T *__restrict__ a, const T *__restrict__ b, T s, T *__restrict__ d, size_t n)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const T x = a[i];
        const T y = SCALAR ? s : b[i];
        T r;
        if (OP == kAdd) r = x + y;
        else if (OP == kSub) r = x - y;
        else if (OP == kMul) r = x * y;
        else if (OP == kDiv) r = x / y;
        else r = s * (T(1) / x);
        d[i] = r;
    }
}

static bool is_device_ptr(const void *p)
{
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

template <typename T, int OP, bool SCALAR>
static cn_status launch_field_op(const T *a, const T *b, T s, T *d, size_t n, cudaStream_t st)
{
    if (n == 0) return CN_OK;
    size_t blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    field_op_kernel<T, OP, SCALAR><<<(unsigned)blocks, 256, 0, st>>>(a, b, s, d, n);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

// Runs one hook synchronously; host operands are staged through device memory.
template <typename T, int OP, bool SCALAR>
static cn_status run_hook(const T *a, const T *b, T s, T *d, size_t n)
{
    if (n == 0) return CN_OK;
    if (!a || !d || (!SCALAR && !b)) return fail(CN_ERR_INVALID_ARGUMENT, "field op: NULL pointer");
    const bool dev = is_device_ptr(a) && is_device_ptr(d) && (SCALAR || is_device_ptr(b));
    if (dev) {
        cn_status r = launch_field_op<T, OP, SCALAR>(a, b, s, d, n, nullptr);
        if (r != CN_OK) return r;
        CN_CUDA_TRY(cudaStreamSynchronize(nullptr));
        return CN_OK;
    }
    T *da = nullptr, *db = nullptr, *dd = nullptr;
    const size_t bytes = n * sizeof(T);
    cudaError_t e = cudaMalloc(&da, bytes);
    if (e == cudaSuccess && !SCALAR) e = cudaMalloc(&db, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&dd, bytes);
    if (e == cudaSuccess) e = cudaMemcpy(da, a, bytes, cudaMemcpyDefault);
    if (e == cudaSuccess && !SCALAR) e = cudaMemcpy(db, b, bytes, cudaMemcpyDefault);
    cn_status r = CN_OK;
    if (e == cudaSuccess) r = launch_field_op<T, OP, SCALAR>(da, db, s, dd, n, nullptr);
    if (e == cudaSuccess && r == CN_OK) e = cudaMemcpy(d, dd, bytes, cudaMemcpyDefault);
    cudaFree(da);
    cudaFree(db);
    cudaFree(dd);
    if (e != cudaSuccess) return cuda_fail(e, "field op staging");
    return r;
}

} // namespace cn

using namespace cn;

#define CN_FIELD2(OPN, OPK, T)                                                            \
    extern "C" void field##OPN##2_##T(const T *src0, const T *src1, T *dst, const size_t n) \
    {                                                                                     \
        (void)run_hook<T, OPK, false>(src0, src1, T(0), dst, n);                          \
    }
#define CN_FIELD1(OPN, OPK, T)                                                            \
    extern "C" void field##OPN##1_##T(const T *src0, const T src1, T *dst, const size_t n) \
    {                                                                                     \
        (void)run_hook<T, OPK, true>(src0, nullptr, src1, dst, n);                        \
    }

CN_FIELD2(Add, kAdd, double)
CN_FIELD2(Sub, kSub, double)
CN_FIELD2(Mul, kMul, double)
CN_FIELD2(Div, kDiv, double)
CN_FIELD2(Add, kAdd, float)
CN_FIELD2(Sub, kSub, float)
CN_FIELD2(Mul, kMul, float)
CN_FIELD2(Div, kDiv, float)
CN_FIELD1(Add, kAdd, double)
CN_FIELD1(Sub, kSub, double)
CN_FIELD1(Mul, kMul, double)
CN_FIELD1(Div, kDiv, double)
CN_FIELD1(Add, kAdd, float)
CN_FIELD1(Sub, kSub, float)
CN_FIELD1(Mul, kMul, float)
CN_FIELD1(Div, kDiv, float)

extern "C" void fieldRcp_double(const double *src0, const double src1, double *dst, const size_t n)
{
    (void)run_hook<double, kRcp, true>(src0, nullptr, src1, dst, n);
}

extern "C" void fieldRcp_float(const float *src0, const float src1, float *dst, const size_t n)
{
    (void)run_hook<float, kRcp, true>(src0, nullptr, src1, dst, n);
}

// Stream-ordered variant on device pointers with a status (same arithmetic).
extern "C" cn_status cn_field_op(int op, cn_dtype dtype, const void *src0, const void *src1,
                                 double scalar, void *dst, size_t n, void *stream)
{
    if (op < kAdd || op > kRcp) return fail(CN_ERR_INVALID_ARGUMENT, "cn_field_op: bad op");
    if (!src0 || !dst)
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_field_op: NULL pointer");
    cudaStream_t st = as_stream(stream);
    const bool sc = (src1 == nullptr);
#define CN_DISPATCH(T)                                                                           \
    {                                                                                            \
        const T *a = (const T *)src0, *b = (const T *)src1;                                      \
        T *d = (T *)dst;                                                                         \
        const T s = (T)scalar;                                                                   \
        switch (op) {                                                                            \
        case kAdd: return sc ? launch_field_op<T, kAdd, true>(a, b, s, d, n, st)                 \
                             : launch_field_op<T, kAdd, false>(a, b, s, d, n, st);               \
        case kSub: return sc ? launch_field_op<T, kSub, true>(a, b, s, d, n, st)                 \
                             : launch_field_op<T, kSub, false>(a, b, s, d, n, st);               \
        case kMul: return sc ? launch_field_op<T, kMul, true>(a, b, s, d, n, st)                 \
                             : launch_field_op<T, kMul, false>(a, b, s, d, n, st);               \
        case kDiv: return sc ? launch_field_op<T, kDiv, true>(a, b, s, d, n, st)                 \
                             : launch_field_op<T, kDiv, false>(a, b, s, d, n, st);               \
        default: return launch_field_op<T, kRcp, true>(a, b, s, d, n, st);                      \
        }                                                                                        \
    }
    if (dtype == CN_FLOAT64) CN_DISPATCH(double)
    if (dtype == CN_FLOAT32) CN_DISPATCH(float)
#undef CN_DISPATCH
    return fail(CN_ERR_UNSUPPORTED, "cn_field_op: dtype must be FLOAT32 or FLOAT64");
}
