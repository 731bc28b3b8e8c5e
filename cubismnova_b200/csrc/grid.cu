// grid.cu -- host side of the C ABI: grid storage, BC vectors, error state.
//
// Grid::Cartesian (Grid/Cartesian.h:50-550) keeps one SoA allocation and hands
// out non-owning block-field views; here the allocation is device memory and
// the views are (component, block) offsets.  Per-field BC vectors
// (Block/Field.h:437-442) live on the host and are flattened into CSR tables
// on the device when a kernel first needs them.
#include "cn_internal.h"
#include "cn_tma.cuh"

#include <cstdio>
#include <cstring>
#include <new>

namespace cn {

static thread_local std::string g_last_error;

cn_status fail(cn_status s, const std::string &msg)
{
    g_last_error = msg;
    return s;
}

cn_status ok() { return CN_OK; }

cn_status grid_check_error(cn_grid *g)
{
    if (!g || !g->d_err) return CN_OK;
    int e = 0;
    CN_CUDA_TRY(cudaMemcpy(&e, g->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e == 0) return CN_OK;
    CN_CUDA_TRY(cudaMemset(g->d_err, 0, sizeof(int)));
    return fail(CN_ERR_DEVICE, "a kernel on this grid gave up a bounded wait (error word " + std::to_string(e) + ")");
}

cn_status cuda_fail(cudaError_t e, const char *what)
{
    std::string m = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) {
        return fail(CN_ERR_OUT_OF_MEMORY, m);
    }
    return fail(CN_ERR_CUDA, m);
}

cn_status check_stencil(const cn_stencil *s)
{
    if (!s) {
        return fail(CN_ERR_INVALID_ARGUMENT, "stencil is NULL");
    }
    // Core/Stencil.h:99-107 compares with Core::Vector's all-components
    // operators (Core/Vector.h:392-421): it throws only if *every* component
    // of begin is > 0, or every component of end is < 1.
    if (s->begin[0] > 0 && s->begin[1] > 0 && s->begin[2] > 0) {
        return fail(CN_ERR_STENCIL_BEGIN, "Stencil: begin_ must be <= 0");
    }
    if (s->end[0] < 1 && s->end[1] < 1 && s->end[2] < 1) {
        return fail(CN_ERR_STENCIL_END, "Stencil: end_ must be > 0");
    }
    for (int d = 0; d < 3; ++d) {
        if (s->begin[d] > 0 || s->end[d] < 1) {
            return fail(CN_ERR_STENCIL_COMPONENT,
                        "Stencil: begin_ must be <= 0 and end_ must be > 0 in every dimension");
        }
    }
    return CN_OK;
}

cn_status check_lab(const cn_grid *g, const cn_stencil *s)
{
    cn_status st = check_stencil(s);
    if (st != CN_OK) {
        return st;
    }
    for (int d = 0; d < 3; ++d) {
        if (-s->begin[d] > g->n[d] || s->end[d] - 1 > g->n[d]) {
            return fail(CN_ERR_STENCIL_TOO_WIDE,
                        "FieldLab: ghost width larger than the block in some dimension");
        }
    }
    return CN_OK;
}

static uint8_t faces_of(const std::vector<HostBC> &v, uint8_t mode)
{
    uint8_t f = 0;
    for (const HostBC &b : v)
        if (b.kind != CN_BC_BASE) f |= (uint8_t)(1u << (2 * b.dir + b.side));
    for (int d = 0; d < 3; ++d) {
        const int c = (mode >> (2 * d)) & 3;
        if (c == 1) f |= (uint8_t)(1u << (2 * d));
        if (c == 2) f |= (uint8_t)(1u << (2 * d + 1));
    }
    return f;
}

static uint8_t mode_of(const std::vector<HostBC> &v)
{
    int periodic[3] = {1, 1, 1};
    int skip[3] = {1, 1, 1};
    for (const HostBC &b : v) {
        periodic[b.dir] = (b.kind == CN_BC_BASE);
        skip[b.dir] = b.side == 0 ? -1 : 1;
    }
    uint8_t m = v.empty() ? 0 : kHasBc;
    for (int d = 0; d < 3; ++d) {
        if (!periodic[d]) {
            m |= (uint8_t)((skip[d] < 0 ? 1 : 2) << (2 * d));
        }
    }
    return m;
}

cn_status sync_bc(cn_grid *g, cudaStream_t stream)
{
    if (!g->bc_dirty) {
        return CN_OK;
    }
    const int nb = g->nblocks;
    std::vector<int32_t> off((size_t)g->ncomp * (nb + 1));
    // mode summaries [comp][block], then face masks [comp][block]
    std::vector<uint8_t> mode((size_t)2 * g->ncomp * nb);
    std::vector<DevBC> ent;
    for (int c = 0; c < g->ncomp; ++c) {
        // offsets are relative to the component's first entry
        const size_t base = ent.size();
        int32_t *o = off.data() + (size_t)c * (nb + 1);
        o[0] = (int32_t)(ent.size() - base);
        for (int b = 0; b < nb; ++b) {
            const auto &v = g->bcs[c][b];
            for (const HostBC &h : v) {
                DevBC d;
                d.meta = h.dir | (h.side << 2) | (h.kind << 3);
                d.pad = 0;
                d.value = h.value;
                ent.push_back(d);
            }
            o[b + 1] = (int32_t)(ent.size() - base);
            mode[(size_t)c * nb + b] = mode_of(v);
            mode[(size_t)(g->ncomp + c) * nb + b] = faces_of(v, mode[(size_t)c * nb + b]);
        }
    }
    // per-component entry bases are folded into separate pointers by bc_view
    // through the offsets table: store the component base in a side vector
    if (ent.empty()) {
        ent.push_back(DevBC{0, 0, 0.0});
    }
    if (ent.size() > g->bc_ent_cap) {
        if (g->d_bc_ent) {
            cudaFree(g->d_bc_ent);
            g->d_bc_ent = nullptr;
        }
        CN_CUDA_TRY(cudaMalloc(&g->d_bc_ent, ent.size() * sizeof(DevBC)));
        g->bc_ent_cap = ent.size();
    }
    // rebase offsets to absolute entry indices
    {
        int32_t acc = 0;
        for (int c = 0; c < g->ncomp; ++c) {
            int32_t *o = off.data() + (size_t)c * (nb + 1);
            const int32_t cnt = o[nb];
            for (int b = 0; b <= nb; ++b) {
                o[b] += acc;
            }
            acc += cnt;
        }
    }
    CN_CUDA_TRY(cudaMemcpyAsync(g->d_bc_ent, ent.data(), ent.size() * sizeof(DevBC),
                                cudaMemcpyHostToDevice, stream));
    CN_CUDA_TRY(cudaMemcpyAsync(g->d_bc_off, off.data(), off.size() * sizeof(int32_t),
                                cudaMemcpyHostToDevice, stream));
    CN_CUDA_TRY(cudaMemcpyAsync(g->d_bc_mode, mode.data(), mode.size(),
                                cudaMemcpyHostToDevice, stream));
    // the host vectors die at scope exit: wait for the pageable copies
    CN_CUDA_TRY(cudaStreamSynchronize(stream));
    g->bc_dirty = false;
    return CN_OK;
}

bool sync_bc_would_allocate(const cn_grid *g)
{
    if (!g->bc_dirty) return false;
    size_t n = 0;
    for (const auto &comp : g->bcs)
        for (const auto &v : comp) n += v.size();
    if (n == 0) n = 1; // an empty table still holds one entry
    return n > g->bc_ent_cap;
}

BcView bc_view(const cn_grid *g, int comp)
{
    BcView v;
    v.off = g->d_bc_off + (size_t)comp * (g->nblocks + 1);
    v.ent = g->d_bc_ent;
    v.mode = g->d_bc_mode + (size_t)comp * g->nblocks;
    v.faces = g->d_bc_mode + (size_t)(g->ncomp + comp) * g->nblocks;
    return v;
}

static size_t dtype_size(cn_dtype t)
{
    switch (t) {
    case CN_FLOAT32:
        return 4;
    case CN_FLOAT64:
        return 8;
    case CN_INT32:
        return 4;
    }
    return 0;
}

} // namespace cn

using namespace cn;

extern "C" {

const char *cn_status_string(cn_status s)
{
    switch (s) {
    case CN_OK: return "ok";
    case CN_ERR_INVALID_ARGUMENT: return "invalid argument";
    case CN_ERR_STENCIL_BEGIN: return "Stencil: begin_ must be <= 0";
    case CN_ERR_STENCIL_END: return "Stencil: end_ must be > 0";
    case CN_ERR_STENCIL_COMPONENT: return "Stencil: begin_ must be <= 0 and end_ must be > 0 in every dimension";
    case CN_ERR_NOT_ALLOCATED: return "FieldLab: can not load lab data when not allocated first";
    case CN_ERR_NO_FIELD: return "FieldLab: no field loaded";
    case CN_ERR_SIZE_MISMATCH: return "Cartesian: Can not assign two grids of unequal size.";
    case CN_ERR_STENCIL_TOO_WIDE: return "FieldLab: ghost width larger than the block in some dimension";
    case CN_ERR_CUDA: return "CUDA error";
    case CN_ERR_OUT_OF_MEMORY: return "out of device memory";
    case CN_ERR_DEVICE: return "device kernel reported an error";
    case CN_ERR_UNSUPPORTED: return "unsupported";
    case CN_ERR_TOO_MANY_BC: return "too many boundary conditions on one block field";
    case CN_ERR_FILE: return "file could not be opened, read or written";
    }
    return "unknown status";
}

const char *cn_last_error_string(void) { return g_last_error.c_str(); }

int cn_abi_version(void) { return CN_ABI_VERSION; }

cn_status cn_device_alloc(size_t bytes, void **ptr)
{
    if (!ptr) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    CN_CUDA_TRY(cudaMalloc(ptr, bytes));
    return CN_OK;
}

cn_status cn_device_free(void *ptr)
{
    if (ptr) CN_CUDA_TRY(cudaFree(ptr));
    return CN_OK;
}

cn_status cn_memcpy(void *dst, const void *src, size_t bytes, void *stream)
{
    if (!dst || !src) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    CN_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, as_stream(stream)));
    if (!stream) CN_CUDA_TRY(cudaStreamSynchronize(nullptr));
    return CN_OK;
}

cn_status cn_stencil_check(const cn_stencil *s) { return check_stencil(s); }

cn_status cn_grid_create(const int nblocks[3], const int block_cells[3], int ncomp,
                         cn_dtype dtype, const double begin[3], const double end[3],
                         cn_grid **out)
{
    return cn_grid_create_entity(nblocks, block_cells, ncomp, dtype, CN_ENTITY_CELL, begin, end, out);
}

// Grid/Cartesian.h:490-513: a block holds cells^3 cell values, (cells+1)^3
// node values, or, per face direction, (cells+1)^3 slots ("slightly more than
// needed") of which the face field's index range (cells + 1 along its
// direction) uses the first ones.
cn_status cn_grid_create_entity(const int nblocks[3], const int block_cells[3], int ncomp, cn_dtype dtype,
                                cn_entity entity, const double begin[3], const double end[3], cn_grid **out)
{
    if (!out || !nblocks || !block_cells) {
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_grid_create: NULL argument");
    }
    *out = nullptr;
    const size_t es = dtype_size(dtype);
    if (es == 0 || ncomp < 1) {
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_grid_create: bad dtype or ncomp");
    }
    if (entity < CN_ENTITY_CELL || entity > CN_ENTITY_FACE_Z) {
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_grid_create: bad entity type");
    }
    int64_t nbl = 1;
    int64_t cells = 1; // storage elements per block
    for (int d = 0; d < 3; ++d) {
        if (nblocks[d] < 1 || block_cells[d] < 1 || block_cells[d] > 1024) {
            return fail(CN_ERR_INVALID_ARGUMENT, "cn_grid_create: block counts and cells must be >= 1");
        }
        nbl *= nblocks[d];
        cells *= block_cells[d] + (entity == CN_ENTITY_CELL ? 0 : 1);
    }
    if (nbl > (1 << 30)) {
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_grid_create: too many blocks");
    }
    cn_grid *g = new (std::nothrow) cn_grid();
    if (!g) {
        return fail(CN_ERR_OUT_OF_MEMORY, "cn_grid_create: host allocation failed");
    }
    g->entity = entity;
    for (int d = 0; d < 3; ++d) {
        g->nb[d] = nblocks[d];
        g->cells[d] = block_cells[d];
        g->n[d] = block_cells[d] + ((entity == CN_ENTITY_NODE || entity == CN_ENTITY_FACE_X + d) ? 1 : 0);
        g->begin[d] = begin ? begin[d] : 0.0;
        g->end[d] = end ? end[d] : 1.0;
        // Mesh/StructuredUniform.h:61: extent / cells
        g->h[d] = (g->end[d] - g->begin[d]) / (double)((int64_t)nblocks[d] * block_cells[d]);
    }
    g->ncomp = ncomp;
    g->dtype = dtype;
    g->esize = es;
    // Grid/Cartesian.h:501-513: block bytes rounded up to 32 bytes
    const size_t bbytes = ((size_t)cells * es + 31) / 32 * 32;
    g->block_stride = (int64_t)(bbytes / es);
    g->nblocks = (int)nbl;
    g->comp_stride = g->block_stride * nbl;
    g->bcs.assign(ncomp, std::vector<std::vector<HostBC>>(nbl));
    g->bc_dirty = false; // the device tables are initialised empty below
    cudaError_t e = cudaGetDevice(&g->device);
    if (e != cudaSuccess) {
        delete g;
        return cuda_fail(e, "cudaGetDevice");
    }
    const size_t total = (size_t)g->comp_stride * ncomp * es;
    e = cudaMalloc(&g->d_data, total);
    if (e == cudaSuccess) e = cudaMemset(g->d_data, 0, total);
    if (e == cudaSuccess) e = cudaMalloc(&g->d_bc_off, sizeof(int32_t) * ncomp * (nbl + 1));
    if (e == cudaSuccess) e = cudaMalloc(&g->d_bc_mode, (size_t)2 * ncomp * nbl);
    if (e == cudaSuccess) e = cudaMalloc(&g->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(g->d_err, 0, sizeof(int));
    // valid empty BC tables from the start: every kernel may read them, even
    // on a grid whose BCs were never pushed or synchronised
    if (e == cudaSuccess) e = cudaMemset(g->d_bc_off, 0, sizeof(int32_t) * ncomp * (nbl + 1));
    if (e == cudaSuccess) e = cudaMemset(g->d_bc_mode, 0, (size_t)2 * ncomp * nbl);
    if (e == cudaSuccess) e = cudaMalloc(&g->d_bc_ent, sizeof(cn::DevBC));
    if (e == cudaSuccess) e = cudaMemset(g->d_bc_ent, 0, sizeof(cn::DevBC));
    if (e == cudaSuccess) g->bc_ent_cap = 1;
    if (e != cudaSuccess) {
        cn_grid_destroy(g);
        return cuda_fail(e, "cn_grid_create allocation");
    }
    *out = g;
    return CN_OK;
}

cn_status cn_grid_destroy(cn_grid *g)
{
    if (!g) {
        return CN_OK;
    }
    if (g->d_data) cudaFree(g->d_data);
    if (g->d_bc_off) cudaFree(g->d_bc_off);
    if (g->d_bc_ent) cudaFree(g->d_bc_ent);
    if (g->d_bc_mode) cudaFree(g->d_bc_mode);
    if (g->d_err) cudaFree(g->d_err);
    delete g;
    return CN_OK;
}

cn_status cn_grid_layout(const cn_grid *g, int64_t *block_stride, int64_t *comp_stride,
                         size_t *total_bytes)
{
    if (!g) {
        return fail(CN_ERR_INVALID_ARGUMENT, "grid is NULL");
    }
    if (block_stride) *block_stride = g->block_stride;
    if (comp_stride) *comp_stride = g->comp_stride;
    if (total_bytes) *total_bytes = (size_t)g->comp_stride * g->ncomp * g->esize;
    return CN_OK;
}

cn_status cn_grid_shape(const cn_grid *g, int info[8])
{
    if (!g || !info) {
        return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    }
    for (int d = 0; d < 3; ++d) {
        info[d] = g->nb[d];
        info[3 + d] = g->n[d];
    }
    info[6] = g->ncomp;
    info[7] = (int)g->dtype;
    return CN_OK;
}

cn_status cn_grid_entity(const cn_grid *g, int *entity, int block_cells[3])
{
    if (!g) return fail(CN_ERR_INVALID_ARGUMENT, "grid is NULL");
    if (entity) *entity = g->entity;
    if (block_cells)
        for (int d = 0; d < 3; ++d) block_cells[d] = g->cells[d];
    return CN_OK;
}

// One CTA waits `polls` times on an mbarrier that nothing completes, as a
// kernel whose TMA copy or tensor-core pipeline never finished would, then
// records the timeout in the error word.
__global__ void wait_timeout_kernel(int polls, int *err)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        bool done = false;
        for (int i = 0; i < polls && !done; ++i) done = mbar_try_wait(&bar, 0);
        if (!done && err) atomicExch(err, kDevErrTimeout);
    }
}

cn_status cn_grid_device_error(cn_grid *g, int *word, int clear)
{
    if (!g || !word) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    CN_CUDA_TRY(cudaDeviceSynchronize());
    CN_CUDA_TRY(cudaMemcpy(word, g->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (clear && *word) CN_CUDA_TRY(cudaMemset(g->d_err, 0, sizeof(int)));
    return CN_OK;
}

cn_status cn_debug_wait_timeout(cn_grid *g, int polls, void *stream)
{
    if (!g || polls < 1 || polls > (1 << 20)) return fail(CN_ERR_INVALID_ARGUMENT, "cn_debug_wait_timeout: bad argument");
    wait_timeout_kernel<<<1, 32, 0, as_stream(stream)>>>(polls, g->d_err);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

cn_status cn_grid_cell_size(const cn_grid *g, double h[3])
{
    if (!g || !h) {
        return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    }
    for (int d = 0; d < 3; ++d) h[d] = g->h[d];
    return CN_OK;
}

cn_status cn_grid_data(cn_grid *g, int comp, void **device_ptr)
{
    if (!g || !device_ptr || comp < 0 || comp >= g->ncomp) {
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_grid_data: bad grid or component");
    }
    *device_ptr = (char *)g->d_data + (size_t)comp * g->comp_stride * g->esize;
    return CN_OK;
}

cn_status cn_grid_upload(cn_grid *g, int comp, const void *host, size_t nbytes, void *stream)
{
    if (!g || !host || comp < 0 || comp >= g->ncomp) {
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_grid_upload: bad grid, component or pointer");
    }
    if (nbytes != (size_t)g->comp_stride * g->esize) {
        return fail(CN_ERR_SIZE_MISMATCH, "cn_grid_upload: byte count does not match the component size");
    }
    void *dst = (char *)g->d_data + (size_t)comp * nbytes;
    CN_CUDA_TRY(cudaMemcpyAsync(dst, host, nbytes, cudaMemcpyHostToDevice, as_stream(stream)));
    return CN_OK;
}

cn_status cn_grid_download(const cn_grid *g, int comp, void *host, size_t nbytes, void *stream)
{
    if (!g || !host || comp < 0 || comp >= g->ncomp) {
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_grid_download: bad grid, component or pointer");
    }
    if (nbytes != (size_t)g->comp_stride * g->esize) {
        return fail(CN_ERR_SIZE_MISMATCH, "cn_grid_download: byte count does not match the component size");
    }
    const void *src = (const char *)g->d_data + (size_t)comp * nbytes;
    CN_CUDA_TRY(cudaMemcpyAsync(host, src, nbytes, cudaMemcpyDeviceToHost, as_stream(stream)));
    return CN_OK;
}

cn_status cn_grid_copy(cn_grid *dst, const cn_grid *src, void *stream)
{
    if (!dst || !src) {
        return fail(CN_ERR_INVALID_ARGUMENT, "grid is NULL");
    }
    if (dst->nblocks != src->nblocks || dst->comp_stride != src->comp_stride ||
        dst->ncomp != src->ncomp || dst->dtype != src->dtype) {
        return fail(CN_ERR_SIZE_MISMATCH, "Cartesian: Can not assign two grids of unequal size.");
    }
    CN_CUDA_TRY(cudaMemcpyAsync(dst->d_data, src->d_data,
                                (size_t)src->comp_stride * src->ncomp * src->esize,
                                cudaMemcpyDeviceToDevice, as_stream(stream)));
    return CN_OK;
}

cn_status cn_bc_push(cn_grid *g, int comp, int block, int dir, int side, cn_bc_kind kind,
                     double value)
{
    if (!g || comp < 0 || comp >= g->ncomp || block < 0 || block >= g->nblocks) {
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_bc_push: bad grid, component or block");
    }
    if (dir < 0 || dir > 2 || side < 0 || side > 1 || kind < CN_BC_BASE || kind > CN_BC_SYMMETRY) {
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_bc_push: bad direction, side or kind");
    }
    auto &v = g->bcs[comp][block];
    if ((int)v.size() >= kMaxBcPerBlock) {
        return fail(CN_ERR_TOO_MANY_BC, "cn_bc_push: BC vector of this block field is full");
    }
    v.push_back(HostBC{dir, side, (int)kind, value});
    g->bc_dirty = true;
    return CN_OK;
}

cn_status cn_bc_push_boundary(cn_grid *g, int comp, int dir, int side, cn_bc_kind kind,
                              double value)
{
    if (!g || dir < 0 || dir > 2 || side < 0 || side > 1) {
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_bc_push_boundary: bad arguments");
    }
    for (int b = 0; b < g->nblocks; ++b) {
        const int bi[3] = {b % g->nb[0], (b / g->nb[0]) % g->nb[1], b / (g->nb[0] * g->nb[1])};
        const bool on_face = side == 0 ? bi[dir] == 0 : bi[dir] == g->nb[dir] - 1;
        if (!on_face) continue;
        cn_status s = cn_bc_push(g, comp, b, dir, side, kind, value);
        if (s != CN_OK) return s;
    }
    return CN_OK;
}

cn_status cn_bc_clear(cn_grid *g, int comp, int block)
{
    if (!g || comp < 0 || comp >= g->ncomp || block < -1 || block >= g->nblocks) {
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_bc_clear: bad grid, component or block");
    }
    if (block < 0) {
        for (auto &v : g->bcs[comp]) v.clear();
    } else {
        g->bcs[comp][block].clear();
    }
    g->bc_dirty = true;
    return CN_OK;
}

cn_status cn_bc_count(const cn_grid *g, int comp, int block, int *count)
{
    if (!g || !count || comp < 0 || comp >= g->ncomp || block < 0 || block >= g->nblocks) {
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_bc_count: bad arguments");
    }
    *count = (int)g->bcs[comp][block].size();
    return CN_OK;
}

cn_status cn_bc_sync(cn_grid *g, void *stream)
{
    if (!g) {
        return fail(CN_ERR_INVALID_ARGUMENT, "grid is NULL");
    }
    return sync_bc(g, as_stream(stream));
}

cn_status cn_lab_extent(const cn_grid *g, const cn_stencil *s, int extent[3])
{
    if (!g || !extent) {
        return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    }
    cn_status st = check_lab(g, s);
    if (st != CN_OK) return st;
    for (int d = 0; d < 3; ++d) extent[d] = g->n[d] - s->begin[d] + s->end[d] - 1;
    return CN_OK;
}

} // extern "C"
