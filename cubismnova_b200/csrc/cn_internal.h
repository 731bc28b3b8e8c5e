// cn_internal.h -- shared host/device definitions of the C-ABI library.
#pragma once

#include "cubismnova_b200.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

namespace cn {

// Largest BC vector per block field.  The reference allows any length; more
// than this many BCs on one block is rejected with CN_ERR_TOO_MANY_BC.
constexpr int kMaxBcPerBlock = 16;

// One BC of a block field as stored on the device (16 bytes).
struct DevBC {
    int32_t meta; // dir | side << 2 | kind << 3
    int32_t pad;
    double value;
};

__host__ __device__ inline int bc_dir(int32_t m) { return m & 3; }
__host__ __device__ inline int bc_side(int32_t m) { return (m >> 2) & 1; }
__host__ __device__ inline int bc_kind(int32_t m) { return (m >> 3) & 7; }

// Per (component, block) summary of the BC vector: bits [2d, 2d+1] hold the
// neighbour skipped in direction d (0: none/periodic, 1: -1 side, 2: +1 side),
// i.e. Block/FieldLab.h:207-214 with the last BC per direction winning.
// Bit 6 is set if the block has any BC at all.
constexpr uint8_t kHasBc = 0x40;

// Device view of the BC tables of one component.
struct BcView {
    const int32_t *off;  // nblocks+1 offsets (CSR)
    const DevBC *ent;    // entries
    const uint8_t *mode; // nblocks summaries
    // nblocks face masks: bit 2d+s set if face (d, s) of the block carries a
    // BC other than Base or its neighbour across that face is skipped; a
    // ghost outside the block across one clear face is the plain periodic
    // neighbour's cell
    const uint8_t *faces;
};

struct HostBC {
    int dir, side, kind;
    double value;
};

} // namespace cn

struct cn_grid {
    int nb[3];
    int n[3];      // block extent in entities: cells, or cells + 1 for nodes / along a face direction
    int cells[3];  // block cells (the mesh)
    int entity;    // cn_entity
    int ncomp;
    cn_dtype dtype;
    double begin[3], end[3], h[3];
    size_t esize;
    int64_t block_stride; // elements
    int64_t comp_stride;  // elements
    int nblocks;
    int device;
    void *d_data;
    // BC vectors [comp][block]
    std::vector<std::vector<std::vector<cn::HostBC>>> bcs;
    bool bc_dirty;
    // device BC tables, component c at c*(nblocks+1) / c*nblocks
    int32_t *d_bc_off;
    cn::DevBC *d_bc_ent;
    uint8_t *d_bc_mode;
    size_t bc_ent_cap;
    int *d_err; // device error word
};

namespace cn {

// thread-local error message handling
cn_status fail(cn_status s, const std::string &msg);
cn_status ok();
cn_status cuda_fail(cudaError_t e, const char *what);
// reads a grid's device error word after the caller synchronised; nonzero:
// CN_ERR_DEVICE (the word is cleared)
cn_status grid_check_error(cn_grid *g);

#define CN_CUDA_TRY(call)                                                      \
    do {                                                                       \
        cudaError_t e__ = (call);                                              \
        if (e__ != cudaSuccess)                                                \
            return ::cn::cuda_fail(e__, #call);                                \
    } while (0)

cn_status check_stencil(const cn_stencil *s);
// Checks stencil validity and that the ghost width fits into a block.
cn_status check_lab(const cn_grid *g, const cn_stencil *s);
// Uploads the BC tables if they changed.
cn_status sync_bc(cn_grid *g, cudaStream_t stream);
// True when sync_bc would have to grow the device BC entry table (cudaMalloc).
bool sync_bc_would_allocate(const cn_grid *g);
BcView bc_view(const cn_grid *g, int comp);

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Runs a set-up step once per device, on the current device: a kernel's
// shared-memory opt-in belongs to each device's context, so a process-wide
// flag would leave the second device without it.  Thread-safe; a failed step
// is retried on the next call.
class DeviceOnce {
  public:
    template <typename F> cn_status run(F &&fn)
    {
        int dev = 0;
        const cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
        if (dev < 0 || dev >= kMaxDevices) return fail(CN_ERR_UNSUPPORTED, "device index out of range");
        std::lock_guard<std::mutex> lk(mu_);
        if (done_[dev]) return CN_OK;
        const cn_status s = fn();
        if (s == CN_OK) done_[dev] = true;
        return s;
    }

  private:
    static constexpr int kMaxDevices = 64;
    std::mutex mu_;
    bool done_[kMaxDevices] = {};
};

// Opts `kernel` into `bytes` of dynamic shared memory, once per device.
template <typename K> inline cn_status smem_opt_in(DeviceOnce &once, K kernel, size_t bytes)
{
    return once.run([&]() -> cn_status {
        CN_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
        return CN_OK;
    });
}

// Geometry of a lab for one stencil on one grid.
struct LabGeom {
    int n[3];  // largest block extent (cells, +1 for nodes / along a face direction)
    int nb[3]; // blocks per dimension
    int lo[3]; // -begin
    int hi[3]; // end - 1
    int tensorial;
    int valid_bc[3]; // BC/Base.h:73-78 per direction
    int64_t bstride;
    // 1 where only the last block along the dimension has extent n and the
    // others n - 1 (node fields: every dimension; face fields: their
    // direction; Grid/BlockFieldAssembler.h:124-135); 0 for cell fields
    int grow[3];
};

// extent along d of the block with coordinate bc along d
__host__ __device__ __forceinline__ int block_extent(const LabGeom &L, int d, int bc)
{
    return L.n[d] - ((L.grow[d] && bc != L.nb[d] - 1) ? 1 : 0);
}

inline LabGeom make_geom(const cn_grid *g, const cn_stencil *s)
{
    LabGeom L;
    for (int d = 0; d < 3; ++d) {
        L.n[d] = g->n[d];
        L.nb[d] = g->nb[d];
        L.lo[d] = -s->begin[d];
        L.hi[d] = s->end[d] - 1;
        L.valid_bc[d] = !(s->begin[d] == 0 || s->end[d] == 1);
    }
    L.tensorial = s->tensorial ? 1 : 0;
    L.bstride = g->block_stride;
    for (int d = 0; d < 3; ++d)
        L.grow[d] = (g->entity == CN_ENTITY_NODE || g->entity == CN_ENTITY_FACE_X + d) ? 1 : 0;
    return L;
}

// ---------------------------------------------------------------------------
// Device: value of lab cell q of block `block` after FieldLab::loadData.
//
// The reference fills a lab in passes (inner copy, 26 neighbour copies, then
// each BC of the vector in order, later BCs overwriting earlier ones).  Here
// every lab cell is resolved on its own: the last BC (highest index k) whose
// slab covers q decides; Dirichlet yields its value, Absorbing and Symmetry
// redirect to a source cell whose value is taken *as it was before BC k ran*,
// i.e. resolved again among BCs 0..k-1.  Each redirect makes the cell inner
// along the BC's direction (ghost width <= block size), so the chain has at
// most 3 links.  With no covering BC the cell holds its loaded value: inner
// data, or the periodic neighbour unless that neighbour was skipped
// (Block/FieldLabLoader.h:196-205).  Returns false if the reference leaves
// the cell undefined.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int pick3(int d, int a, int b, int c) { return d == 0 ? a : (d == 1 ? b : c); }

// GROW: the grid may hold node / face fields (per-block extents); cell grids
// (every fused stencil kernel) compile without that logic.  The resolution
// ends in the sink: sink.value(v) for a Dirichlet value (the chain's signs
// applied), sink.load(idx, nsign, s0, s1, s2) for comp[idx] times the chain's
// signs, innermost first.  lab_value's sink loads at once; a kernel can
// instead collect several cells' sources and issue their loads together.
template <typename T, bool GROW, typename Sink>
__device__ __forceinline__ bool lab_resolve(const LabGeom &L, const BcView &bc, uint8_t mode, int block, int bx,
                                            int by, int bz, int q0, int q1, int q2, bool apply_bc, Sink &sink)
{
    // this block's extents (node / face fields: the last block along a grown
    // dimension holds one more entity); cells past its lab range are not part
    // of its lab
    const int e0 = GROW ? block_extent(L, 0, bx) : L.n[0];
    const int e1 = GROW ? block_extent(L, 1, by) : L.n[1];
    const int e2 = GROW ? block_extent(L, 2, bz) : L.n[2];
    if (GROW && (q0 >= e0 + L.hi[0] || q1 >= e1 + L.hi[1] || q2 >= e2 + L.hi[2]))
        return false;
    // skip flags hold even when the BCs themselves are not applied
    T s0 = T(1), s1 = T(1), s2 = T(1); // symmetry signs of the chain, outermost first
    int nsign = 0;
    if (apply_bc && (mode & kHasBc)) {
        const int k0 = bc.off[block];
        int kmax = bc.off[block + 1] - k0;
        const DevBC *e = bc.ent + k0;
        for (int link = 0; link < 4; ++link) {
            int found = -1;
            int32_t meta = 0;
            for (int k = kmax - 1; k >= 0; --k) {
                const int32_t m = e[k].meta;
                if (bc_kind(m) == CN_BC_BASE)
                    continue;
                const int d = bc_dir(m);
                if (!pick3(d, L.valid_bc[0], L.valid_bc[1], L.valid_bc[2]))
                    continue;
                const int qd = pick3(d, q0, q1, q2);
                const int nd = pick3(d, e0, e1, e2);
                if (!(bc_side(m) == 0 ? (qd < 0) : (qd >= nd)))
                    continue;
                if (!L.tensorial) {
                    const bool in0 = d == 0 || ((unsigned)q0 < (unsigned)e0);
                    const bool in1 = d == 1 || ((unsigned)q1 < (unsigned)e1);
                    const bool in2 = d == 2 || ((unsigned)q2 < (unsigned)e2);
                    if (!(in0 && in1 && in2))
                        continue;
                }
                found = k;
                meta = m;
                break;
            }
            if (found < 0)
                break;
            const int d = bc_dir(meta);
            const int kind = bc_kind(meta);
            const int nd = pick3(d, e0, e1, e2);
            if (kind == CN_BC_DIRICHLET) {
                T v = static_cast<T>(e[found].value);
                // apply the chain's signs innermost first
                if (nsign > 2) v = s2 * v;
                if (nsign > 1) v = s1 * v;
                if (nsign > 0) v = s0 * v;
                sink.value(v);
                return true;
            }
            int qd = pick3(d, q0, q1, q2);
            if (kind == CN_BC_ABSORBING) {
                qd = bc_side(meta) == 0 ? 0 : nd - 1;
            } else { // symmetry: r = roffset - q
                qd = (bc_side(meta) == 0 ? -1 : 2 * nd - 1) - qd;
                const T sg = static_cast<T>(e[found].value);
                if (nsign == 0) s0 = sg;
                else if (nsign == 1) s1 = sg;
                else s2 = sg;
                ++nsign;
            }
            if (d == 0) q0 = qd;
            else if (d == 1) q1 = qd;
            else q2 = qd;
            kmax = found;
        }
    }
    // loaded value
    const int r0 = q0 < 0 ? -1 : (q0 >= e0 ? 1 : 0);
    const int r1 = q1 < 0 ? -1 : (q1 >= e1 ? 1 : 0);
    const int r2 = q2 < 0 ? -1 : (q2 >= e2 ? 1 : 0);
    int src_block = block;
    int s0e = e0, s1e = e1; // extents (x, y) of the source block
    if (r0 | r1 | r2) {
        if (!L.tensorial && (r0 != 0) + (r1 != 0) + (r2 != 0) > 1)
            return false;
        // skipped neighbour: Block/FieldLab.h:207-214 + FieldLabLoader.h:197-201
        const int c0 = mode & 3, c1 = (mode >> 2) & 3, c2 = (mode >> 4) & 3;
        if ((r0 != 0 && c0 == (r0 < 0 ? 1 : 2)) || (r1 != 0 && c1 == (r1 < 0 ? 1 : 2)) ||
            (r2 != 0 && c2 == (r2 < 0 ? 1 : 2)))
            return false;
        int nbx = bx + r0, nby = by + r1, nbz = bz + r2;
        nbx = nbx < 0 ? nbx + L.nb[0] : (nbx >= L.nb[0] ? nbx - L.nb[0] : nbx);
        nby = nby < 0 ? nby + L.nb[1] : (nby >= L.nb[1] ? nby - L.nb[1] : nby);
        nbz = nbz < 0 ? nbz + L.nb[2] : (nbz >= L.nb[2] ? nbz - L.nb[2] : nbz);
        src_block = nbx + L.nb[0] * (nby + L.nb[1] * nbz);
        // a lower neighbour is read from its end (its own extent), an upper
        // one from its start (FieldLabLoader.h:212-214, 230-240)
        const int ne0 = GROW ? block_extent(L, 0, nbx) : L.n[0];
        const int ne1 = GROW ? block_extent(L, 1, nby) : L.n[1];
        const int ne2 = GROW ? block_extent(L, 2, nbz) : L.n[2];
        q0 += r0 < 0 ? ne0 : -r0 * e0;
        q1 += r1 < 0 ? ne1 : -r1 * e1;
        q2 += r2 < 0 ? ne2 : -r2 * e2;
        s0e = ne0;
        s1e = ne1;
    }
    sink.load((int64_t)src_block * L.bstride + q0 + (int64_t)s0e * (q1 + (int64_t)s1e * q2), nsign, s0, s1, s2);
    return true;
}

// the sink of lab_value: the value at once
template <typename T> struct LabLoad {
    const T *__restrict__ comp;
    T &out;
    __device__ __forceinline__ void value(T v) { out = v; }
    __device__ __forceinline__ void load(int64_t idx, int nsign, T s0, T s1, T s2)
    {
        T v = comp[idx];
        if (nsign > 2) v = s2 * v;
        if (nsign > 1) v = s1 * v;
        if (nsign > 0) v = s0 * v;
        out = v;
    }
};

template <typename T, bool GROW = false>
__device__ __forceinline__ bool lab_value(const T *__restrict__ comp, const LabGeom &L,
                                          const BcView &bc, int block, int bx, int by, int bz,
                                          int q0, int q1, int q2, bool apply_bc, T &out)
{
    LabLoad<T> sink{comp, out};
    return lab_resolve<T, GROW>(L, bc, bc.mode[block], block, bx, by, bz, q0, q1, q2, apply_bc, sink);
}

// Lab value through the full BC chain (out of line: only blocks with BCs or
// skip flags take it, so its code exists once per kernel; kernels calling it
// pass L and bc from __grid_constant__ parameters or device memory).
template <typename T>
__device__ __noinline__ T lab_fetch_slow(const T *comp, const LabGeom &L, const BcView &bc, int block, int x, int y,
                                    int z)
{
    const int bx = block % L.nb[0];
    const int by = (block / L.nb[0]) % L.nb[1];
    const int bz = block / (L.nb[0] * L.nb[1]);
    T v;
    if (!lab_value<T>(comp, L, bc, block, bx, by, bz, x, y, z, true, v))
        v = T(0);
    return v;
}

// Value of component comp at cell (x,y,z) of `block` (may lie outside it);
// cell-centred grids (every block has extent L.n): in-block cells and the periodic neighbours of blocks without BCs
// or skip flags (lab mode byte 0, what cn::lab_value resolves to for them)
// are plain loads; the rest go through the lab.
template <typename T>
__device__ __forceinline__ T lab_fetch(const T *comp, const LabGeom &L, const BcView &bc, int block,
                                   int x, int y, int z)
{
    if ((unsigned)x < (unsigned)L.n[0] && (unsigned)y < (unsigned)L.n[1] &&
        (unsigned)z < (unsigned)L.n[2])
        return __ldg(comp + (int64_t)block * L.bstride + x + (int64_t)L.n[0] * (y + (int64_t)L.n[1] * z));
    if (__ldg(bc.mode + block) != 0)
        return lab_fetch_slow<T>(comp, L, bc, block, x, y, z);
    const int r0 = x < 0 ? -1 : (x >= L.n[0] ? 1 : 0);
    const int r1 = y < 0 ? -1 : (y >= L.n[1] ? 1 : 0);
    const int r2 = z < 0 ? -1 : (z >= L.n[2] ? 1 : 0);
    if (!L.tensorial && (r0 != 0) + (r1 != 0) + (r2 != 0) > 1)
        return T(0); // outside a non-tensorial lab: undefined, read as 0
    int nbx = block % L.nb[0] + r0, nby = (block / L.nb[0]) % L.nb[1] + r1, nbz = block / (L.nb[0] * L.nb[1]) + r2;
    nbx = nbx < 0 ? nbx + L.nb[0] : (nbx >= L.nb[0] ? nbx - L.nb[0] : nbx);
    nby = nby < 0 ? nby + L.nb[1] : (nby >= L.nb[1] ? nby - L.nb[1] : nby);
    nbz = nbz < 0 ? nbz + L.nb[2] : (nbz >= L.nb[2] ? nbz - L.nb[2] : nbz);
    const int src = nbx + L.nb[0] * (nby + L.nb[1] * nbz);
    x -= r0 * L.n[0];
    y -= r1 * L.n[1];
    z -= r2 * L.n[2];
    return __ldg(comp + (int64_t)src * L.bstride + x + (int64_t)L.n[0] * (y + (int64_t)L.n[1] * z));
}

} // namespace cn
