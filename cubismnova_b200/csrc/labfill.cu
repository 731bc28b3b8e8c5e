// labfill.cu -- K0: explicit lab fill (Cartesian::loadLab into lab buffers).
//
// One thread per lab cell; each cell is resolved independently by
// cn::lab_value (inner copy, periodic neighbour gather, BC chain).  Writes are
// coalesced along x of the lab; reads of inner and face cells are coalesced
// along x of the source block.  This kernel exists so the device ghost fill
// can be compared with the reference FieldLab bit for bit; the stencil
// kernels fuse the same resolution into their shared-memory staging.
#include "cn_internal.h"

namespace cn {

template <typename T, bool GROW>
__global__ void __launch_bounds__(256)
    lab_fill_kernel(const T *__restrict__ comp, LabGeom L, BcView bc, int block_begin,
                    int block_count, int apply_bc, T *__restrict__ out)
{
    const int E0 = L.n[0] + L.lo[0] + L.hi[0];
    const int E1 = L.n[1] + L.lo[1] + L.hi[1];
    const int E2 = L.n[2] + L.lo[2] + L.hi[2];
    const int64_t lab_cells = (int64_t)E0 * E1 * E2;
    const int64_t total = lab_cells * block_count;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int bl = (int)(t / lab_cells);
        const int64_t c = t - (int64_t)bl * lab_cells;
        const int x = (int)(c % E0);
        const int y = (int)((c / E0) % E1);
        const int z = (int)(c / ((int64_t)E0 * E1));
        const int block = block_begin + bl;
        const int bx = block % L.nb[0];
        const int by = (block / L.nb[0]) % L.nb[1];
        const int bz = block / (L.nb[0] * L.nb[1]);
        T v;
        if (lab_value<T, GROW>(comp, L, bc, block, bx, by, bz, x - L.lo[0], y - L.lo[1],
                               z - L.lo[2], apply_bc != 0, v)) {
            out[t] = v;
        }
    }
}

template <typename T>
static cn_status launch_fill(cn_grid *g, int comp, const cn_stencil *s, int b0, int cnt,
                             int apply_bc, void *d_labs, cudaStream_t st)
{
    const LabGeom L = make_geom(g, s);
    const T *src = reinterpret_cast<const T *>(g->d_data) + (size_t)comp * g->comp_stride;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
    const int64_t E = (int64_t)(L.n[0] + L.lo[0] + L.hi[0]) * (L.n[1] + L.lo[1] + L.hi[1]) *
                      (L.n[2] + L.lo[2] + L.hi[2]);
    const int64_t total = E * cnt;
    int64_t blocks = (total + 255) / 256;
    const int64_t cap = (int64_t)sms * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    if (L.grow[0] || L.grow[1] || L.grow[2])
        lab_fill_kernel<T, true><<<(unsigned)blocks, 256, 0, st>>>(src, L, bc_view(g, comp), b0, cnt, apply_bc,
                                                                   reinterpret_cast<T *>(d_labs));
    else
        lab_fill_kernel<T, false><<<(unsigned)blocks, 256, 0, st>>>(src, L, bc_view(g, comp), b0, cnt, apply_bc,
                                                                    reinterpret_cast<T *>(d_labs));
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

} // namespace cn

using namespace cn;

extern "C" cn_status cn_lab_fill(cn_grid *g, int comp, const cn_stencil *s, int block_begin,
                                 int block_count, int apply_bc, void *d_labs, void *stream)
{
    if (!g) {
        return fail(CN_ERR_NOT_ALLOCATED, "FieldLab: can not load lab data when not allocated first");
    }
    if (comp < 0 || comp >= g->ncomp) {
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_lab_fill: bad component");
    }
    if (!d_labs) {
        return fail(CN_ERR_NOT_ALLOCATED, "FieldLab: can not load lab data when not allocated first");
    }
    cn_status st = check_lab(g, s);
    if (st != CN_OK) return st;
    if (block_begin < 0 || block_count < 0 || block_begin + (int64_t)block_count > g->nblocks) {
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_lab_fill: block range outside the grid");
    }
    if (block_count == 0) return CN_OK;
    cudaStream_t cs = as_stream(stream);
    st = sync_bc(g, cs);
    if (st != CN_OK) return st;
    switch (g->dtype) {
    case CN_FLOAT64:
        return launch_fill<double>(g, comp, s, block_begin, block_count, apply_bc, d_labs, cs);
    case CN_FLOAT32:
        return launch_fill<float>(g, comp, s, block_begin, block_count, apply_bc, d_labs, cs);
    case CN_INT32:
        return launch_fill<int32_t>(g, comp, s, block_begin, block_count, apply_bc, d_labs, cs);
    }
    return fail(CN_ERR_UNSUPPORTED, "cn_lab_fill: dtype");
}
