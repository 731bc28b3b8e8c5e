// aos.cu -- grid <-> array-of-structures (AoS) file buffer on the device.
//
// The reference writes a grid to a file by copying every block field into
// one AoS buffer in a host loop over blocks (IO/CartesianHDF.h:76-80, OpenMP
// over blocks) with Field2AOS (IO/FieldAOS.h:37-57 scalar, :79-101 tensor,
// :136-141 face container -> the face field of one direction), and reads it
// back with AOS2Field (:59-77, :103-124).  For a file index range r (global
// entity indices, the HDF dataset's hyperslab) and every point p of r that
// lies in the grid:
//     buf[c + ncomp * flat_r(p)] = (FileT) field_c[p]       (Field2AOS)
//     field_c[p] = (T) buf[c + ncomp * flat_r(p)]           (AOS2Field)
// with flat_r the x-fastest flat index over r's extent; points of r outside
// the grid are not touched.  Here one launch covers the whole grid: a CTA
// takes a chunk of up to kPts points of one x-row of the intersection, reads
// each component with coalesced loads (consecutive x are consecutive in a
// block), converts, interleaves the components in shared memory and writes
// the chunk's ncomp * len contiguous file values with coalesced stores (the
// reverse for the read).  HBM-bound: ncomp * (sizeof(T) + sizeof(FileT))
// bytes per point.
#include "cn_fastdiv.h"
#include "cn_internal.h"

namespace cn {
namespace aos {

constexpr int kThreads = 256;             // threads per CTA
constexpr int kPer = 2;                   // points per thread and work item
constexpr int kPts = kThreads * kPer;     // points per work item (one x-row chunk)
constexpr int kMaxComp = 16;              // components per call
constexpr size_t kSmemDefault = 48 << 10; // above this the kernel opts in

struct Geo {
    int nb[3];       // blocks
    int cells[3];    // block cells
    int grow[3];     // 1: the last block along d holds cells + 1 entities
    int ib[3];       // intersection begin (global entity index)
    int ie[3];       // intersection extent
    int sb[3];       // file range begin
    int se[3];       // file range extent
    int comp0, ncomp;
    int chunks;      // kPts chunks per x-row of the intersection
    int items;       // rows * chunks
    FastDiv dv_chunks, dv_ie1, dv_c0, dv_c1, dv_c2;
    int64_t bstride; // elements
    int64_t cstride; // elements
};

template <typename D, typename S> __device__ __forceinline__ D conv(S v) { return static_cast<D>(v); }

// One work item is up to kPts consecutive points of one x-row of the
// intersection; a thread takes points t and t + kThreads.  All divisions are
// multiply-high forms of divisors fixed at launch (cn_fastdiv.h).  MAXC >= ncomp
// bounds the component loops at compile time so that a thread issues every
// load of its points before converting any.
// The item's file values dst[0, n) <-> shared st[0, n): 16-byte accesses
// when dst is 16-byte aligned and n * sizeof(F) a multiple of 16 (whole-grid
// files with 4-byte values and 4 | x-extent * ncomp, or 8-byte values and
// 2 | it), else element by element.
template <typename F, bool OUT>
__device__ __forceinline__ void stage_copy(F *dst, F *st, int n, int t)
{
    const size_t bytes = (size_t)n * sizeof(F);
    if ((reinterpret_cast<uintptr_t>(dst) & 15) == 0 && (bytes & 15) == 0) {
        int4 *d4 = reinterpret_cast<int4 *>(dst);
        int4 *s4 = reinterpret_cast<int4 *>(st);
        const int n4 = (int)(bytes >> 4);
        for (int k = t; k < n4; k += kThreads) {
            if (OUT) d4[k] = s4[k];
            else s4[k] = __ldg(d4 + k);
        }
    } else {
        for (int k = t; k < n; k += kThreads) {
            if (OUT) dst[k] = st[k];
            else st[k] = __ldg(dst + k);
        }
    }
}

// Resident CTAs per SM that the register budget is set for (every
// instantiation compiles without spills at these bounds).
constexpr int min_ctas(bool to_aos, int maxc)
{
    return maxc > 4 ? 2 : (to_aos ? (maxc == 1 ? 8 : 6) : (maxc == 1 ? 6 : 5));
}

template <typename T, typename F, bool TO_AOS, int MAXC>
__global__ void __launch_bounds__(kThreads, min_ctas(TO_AOS, MAXC))
    aos_kernel(const __grid_constant__ Geo G, T *__restrict__ grid, F *__restrict__ buf)
{
    extern __shared__ __align__(16) unsigned char aos_smem[];
    F *st = reinterpret_cast<F *>(aos_smem);
    const int t = threadIdx.x;
    const int nc = G.ncomp;
    T *const gbase = grid + (int64_t)G.comp0 * G.cstride;
    for (int w = blockIdx.x; w < G.items; w += gridDim.x) {
        const int row = G.dv_chunks.div(w);
        const int chunk = w - row * G.chunks;
        const int iz = G.dv_ie1.div(row);
        const int gy = G.ib[1] + (row - iz * G.ie[1]);
        const int gz = G.ib[2] + iz;
        const int by = min(G.dv_c1.div(gy), G.nb[1] - 1), ly = gy - by * G.cells[1];
        const int bz = min(G.dv_c2.div(gz), G.nb[2] - 1), lz = gz - bz * G.cells[2];
        const int ey = G.cells[1] + ((G.grow[1] && by == G.nb[1] - 1) ? 1 : 0);
        const int rowblk = G.nb[0] * (by + G.nb[1] * bz); // block index of the row's x = 0 block
        const int inrow = ly + ey * lz;                    // (y, z) row inside its block
        const int xs = chunk * kPts;                       // item start, relative to ib[0]
        const int len = min(kPts, G.ie[0] - xs);
        F *dst = buf + ((int64_t)(G.ib[0] + xs - G.sb[0]) +
                        (int64_t)G.se[0] * ((gy - G.sb[1]) + (int64_t)G.se[1] * (gz - G.sb[2]))) * nc;
        // in-grid offset of point p of the item
        auto offset = [&](int p) -> int64_t {
            const int x = G.ib[0] + xs + p;
            const int bx = min(G.dv_c0.div(x), G.nb[0] - 1), lx = x - bx * G.cells[0];
            const int ex = G.cells[0] + ((G.grow[0] && bx == G.nb[0] - 1) ? 1 : 0);
            return (int64_t)(bx + rowblk) * G.bstride + lx + (int64_t)ex * inrow;
        };
        if (TO_AOS) {
            T v[kPer][MAXC];
#pragma unroll
            for (int j = 0; j < kPer; ++j) {
                if (t + j * kThreads < len) {
                    const int64_t off = offset(t + j * kThreads);
#pragma unroll
                    for (int c = 0; c < MAXC; ++c)
                        if (c < nc) v[j][c] = __ldg(gbase + off + c * G.cstride);
                }
            }
#pragma unroll
            for (int j = 0; j < kPer; ++j) {
                const int p = t + j * kThreads;
                if (p < len) {
#pragma unroll
                    for (int c = 0; c < MAXC; ++c)
                        if (c < nc) st[p * nc + c] = conv<F>(v[j][c]);
                }
            }
            __syncthreads();
            stage_copy<F, true>(dst, st, len * nc, t);
        } else {
            stage_copy<F, false>(dst, st, len * nc, t);
            __syncthreads();
#pragma unroll
            for (int j = 0; j < kPer; ++j) {
                const int p = t + j * kThreads;
                if (p < len) {
                    const int64_t off = offset(p);
#pragma unroll
                    for (int c = 0; c < MAXC; ++c)
                        if (c < nc) gbase[off + c * G.cstride] = conv<T>(st[p * nc + c]);
                }
            }
        }
        __syncthreads();
    }
}

template <typename T, typename F, bool TO_AOS, int MAXC>
cn_status launch_one(const Geo &G, T *data, F *buf, size_t smem, int grid, cudaStream_t s)
{
    // the opt-in is a property of the current device's context: set it on every large launch
    if (smem > kSmemDefault) {
        CN_CUDA_TRY(cudaFuncSetAttribute(aos_kernel<T, F, TO_AOS, MAXC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(kPts * kMaxComp * sizeof(F))));
    }
    aos_kernel<T, F, TO_AOS, MAXC><<<grid, kThreads, smem, s>>>(G, data, buf);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

template <typename T, typename F>
cn_status launch(const Geo &G, cn_grid *g, void *buf, bool to_aos, cudaStream_t s)
{
    int dev = 0, nsm = 0;
    CN_CUDA_TRY(cudaGetDevice(&dev));
    CN_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    // up to 8 resident CTAs of 256 threads per SM, grid-stride over the items
    const int grid = G.items < nsm * 8 ? G.items : nsm * 8;
    const size_t smem = (size_t)kPts * G.ncomp * sizeof(F);
    T *data = reinterpret_cast<T *>(g->d_data);
    F *b = reinterpret_cast<F *>(buf);
    const int nc = G.ncomp;
    if (to_aos) {
        if (nc == 1) return launch_one<T, F, true, 1>(G, data, b, smem, grid, s);
        if (nc <= 4) return launch_one<T, F, true, 4>(G, data, b, smem, grid, s);
        return launch_one<T, F, true, kMaxComp>(G, data, b, smem, grid, s);
    }
    if (nc == 1) return launch_one<T, F, false, 1>(G, data, b, smem, grid, s);
    if (nc <= 4) return launch_one<T, F, false, 4>(G, data, b, smem, grid, s);
    return launch_one<T, F, false, kMaxComp>(G, data, b, smem, grid, s);
}

template <typename T>
cn_status dispatch_file(const Geo &G, cn_grid *g, cn_dtype file_dtype, void *buf, bool to_aos, cudaStream_t s)
{
    switch (file_dtype) {
    case CN_FLOAT64:
        return launch<T, double>(G, g, buf, to_aos, s);
    case CN_FLOAT32:
        return launch<T, float>(G, g, buf, to_aos, s);
    case CN_INT32:
        return launch<T, int32_t>(G, g, buf, to_aos, s);
    }
    return fail(CN_ERR_UNSUPPORTED, "cn_grid_aos: file dtype");
}

cn_status run(cn_grid *g, int comp0, int ncomp, const int span_begin[3], const int span_end[3],
              cn_dtype file_dtype, void *buf, void *stream, bool to_aos)
{
    const char *who = to_aos ? "cn_grid_to_aos" : "cn_grid_from_aos";
    if (!g || !span_begin || !span_end) {
        return fail(CN_ERR_INVALID_ARGUMENT, std::string(who) + ": grid or file range is NULL");
    }
    if (comp0 < 0 || ncomp < 1 || comp0 + ncomp > g->ncomp) {
        return fail(CN_ERR_INVALID_ARGUMENT, std::string(who) + ": components outside the grid");
    }
    if (ncomp > kMaxComp) {
        return fail(CN_ERR_UNSUPPORTED, std::string(who) + ": more than 16 components per call");
    }
    if (file_dtype < CN_FLOAT32 || file_dtype > CN_INT32) {
        return fail(CN_ERR_INVALID_ARGUMENT, std::string(who) + ": bad file dtype");
    }
    // a floating-point value converted to int32 is undefined out of range in
    // the reference's implicit conversion; only int32 <-> int32 is allowed
    const cn_dtype dst_type = to_aos ? file_dtype : g->dtype;
    const cn_dtype src_type = to_aos ? g->dtype : file_dtype;
    if (dst_type == CN_INT32 && src_type != CN_INT32) {
        return fail(CN_ERR_UNSUPPORTED, std::string(who) + ": floating-point to int32 conversion");
    }
    Geo G;
    int64_t rows = 1;
    for (int d = 0; d < 3; ++d) {
        if (span_end[d] < span_begin[d]) {
            return fail(CN_ERR_INVALID_ARGUMENT, std::string(who) + ": file range end before begin");
        }
        G.nb[d] = g->nb[d];
        G.cells[d] = g->cells[d];
        G.grow[d] = (g->entity == CN_ENTITY_NODE || g->entity == CN_ENTITY_FACE_X + d) ? 1 : 0;
        G.sb[d] = span_begin[d];
        G.se[d] = span_end[d] - span_begin[d];
        // grid index range [0, nb * cells + grow)
        const int gend = g->nb[d] * g->cells[d] + G.grow[d];
        const int b = span_begin[d] > 0 ? span_begin[d] : 0;
        const int e = span_end[d] < gend ? span_end[d] : gend;
        G.ib[d] = b;
        G.ie[d] = e > b ? e - b : 0;
        if (d > 0) rows *= G.ie[d];
    }
    if ((int64_t)G.se[0] * G.se[1] * G.se[2] > 0 && !buf) {
        return fail(CN_ERR_INVALID_ARGUMENT, std::string(who) + ": buffer is NULL");
    }
    if (G.ie[0] == 0 || rows == 0) return CN_OK; // empty intersection
    // the kernel dereferences buf: device, managed or pinned host memory only
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, buf) != cudaSuccess || pa.type == cudaMemoryTypeUnregistered) {
        cudaGetLastError();
        return fail(CN_ERR_INVALID_ARGUMENT, std::string(who) + ": buffer is not device-accessible memory");
    }
    G.comp0 = comp0;
    G.ncomp = ncomp;
    G.chunks = (G.ie[0] + kPts - 1) / kPts;
    if (rows * G.chunks >= (int64_t(1) << 31)) {
        return fail(CN_ERR_UNSUPPORTED, std::string(who) + ": more than 2^31 row chunks in the file range");
    }
    G.items = (int)(rows * G.chunks);
    G.dv_chunks = FastDiv((uint32_t)G.chunks);
    G.dv_ie1 = FastDiv((uint32_t)G.ie[1]);
    G.dv_c0 = FastDiv((uint32_t)G.cells[0]);
    G.dv_c1 = FastDiv((uint32_t)G.cells[1]);
    G.dv_c2 = FastDiv((uint32_t)G.cells[2]);
    G.bstride = g->block_stride;
    G.cstride = g->comp_stride;
    cudaStream_t s = as_stream(stream);
    switch (g->dtype) {
    case CN_FLOAT64:
        return dispatch_file<double>(G, g, file_dtype, buf, to_aos, s);
    case CN_FLOAT32:
        return dispatch_file<float>(G, g, file_dtype, buf, to_aos, s);
    case CN_INT32:
        return dispatch_file<int32_t>(G, g, file_dtype, buf, to_aos, s);
    }
    return fail(CN_ERR_UNSUPPORTED, std::string(who) + ": grid dtype");
}

} // namespace aos
} // namespace cn

extern "C" cn_status cn_grid_to_aos(cn_grid *g, int comp0, int ncomp, const int span_begin[3],
                                    const int span_end[3], cn_dtype file_dtype, void *d_buf, void *stream)
{
    return cn::aos::run(g, comp0, ncomp, span_begin, span_end, file_dtype, d_buf, stream, true);
}

extern "C" cn_status cn_grid_from_aos(cn_grid *g, int comp0, int ncomp, const int span_begin[3],
                                      const int span_end[3], cn_dtype file_dtype, const void *d_buf, void *stream)
{
    return cn::aos::run(g, comp0, ncomp, span_begin, span_end, file_dtype, const_cast<void *>(d_buf), stream,
                        false);
}
