// cubismnova_b200.hpp -- C++ facade of the C ABI with the reference's names.
//
// Header-only: a reference user includes this instead of Cubism/Grid/Cartesian.h,
// Cubism/Block/FieldLab.h, Cubism/BC/*.h and Cubism/Core/Stencil.h and links
// libcubismnova_b200.so.  Class and method names, argument meaning and the
// exception messages follow CubismNova; the data lives on the GPU:
//
//   Grid::Cartesian<T>     Grid/Cartesian.h:50-550 (device SoA, same layout)
//   Grid::BlockField<T>    the block field views of Grid/Cartesian.h:334-373
//                          with getBC() (Block/Field.h:437-442)
//   Block::FieldLab<T>     Block/FieldLab.h:30-492 (allocate, loadData,
//                          active ranges, getActiveField, footprint)
//   BC::Base/Dirichlet/Absorbing/Symmetry   BC/*.h
//   Core::Stencil          Core/Stencil.h:21-108
//   Ops::laplacian/gradient/lapGrad/divergence   the benchmark stencils
//   IO::Field2AOS/AOS2Field/gatherAOS   IO/FieldAOS.h over every block
//   IO::CartesianWriteHDF/ReadHDF       IO/CartesianHDF.h (HDF5 files written by the library)
//
// Errors raise std::runtime_error with the reference's message where the
// reference throws (Core/Stencil.h:101-106, Block/FieldLab.h:189-190,
// :417-419, Grid/Cartesian.h:162-164).
#pragma once

#include "cubismnova_b200.h"

#include <array>
#include <cstddef>
#include <cstdio>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace cubism_b200 {

inline void check(cn_status s)
{
    if (s != CN_OK) {
        const char *m = cn_last_error_string();
        throw std::runtime_error((m && *m) ? std::string(m) : std::string(cn_status_string(s)));
    }
}

template <typename T> struct DType;
template <> struct DType<double> { static constexpr cn_dtype value = CN_FLOAT64; };
template <> struct DType<float> { static constexpr cn_dtype value = CN_FLOAT32; };
template <> struct DType<int> { static constexpr cn_dtype value = CN_INT32; };

using MultiIndex = std::array<int, 3>;

namespace Core {
/// Core::Stencil(begin, end, tensorial): begin <= 0 inclusive, end > 0 exclusive.
class Stencil {
public:
    Stencil() : Stencil(0, 1, false) {}
    Stencil(int b, int e, bool tensorial = false) : Stencil(MultiIndex{b, b, b}, MultiIndex{e, e, e}, tensorial) {}
    Stencil(const MultiIndex &b, const MultiIndex &e, bool tensorial = false)
    {
        for (int d = 0; d < 3; ++d) {
            s_.begin[d] = b[d];
            s_.end[d] = e[d];
        }
        s_.tensorial = tensorial ? 1 : 0;
        check(cn_stencil_check(&s_));
    }
    MultiIndex getBegin() const { return {s_.begin[0], s_.begin[1], s_.begin[2]}; }
    MultiIndex getEnd() const { return {s_.end[0], s_.end[1], s_.end[2]}; }
    bool isTensorial() const { return s_.tensorial != 0; }
    const cn_stencil *raw() const { return &s_; }

private:
    cn_stencil s_;
};

/// The subset of Core::IndexRange used by the lab API (begin inclusive, end exclusive).
struct IndexRange {
    MultiIndex begin{0, 0, 0}, end{0, 0, 0};
    MultiIndex getBegin() const { return begin; }
    MultiIndex getEnd() const { return end; }
    MultiIndex getExtent() const { return {end[0] - begin[0], end[1] - begin[1], end[2] - begin[2]}; }
    size_t size() const
    {
        const MultiIndex e = getExtent();
        return (size_t)e[0] * e[1] * e[2];
    }
};
} // namespace Core

namespace BC {
/// BC::Base (periodic no-op) and the three concrete BCs (BC/Base.h:39-79).
struct Base {
    Base(size_t dir, size_t side) : dir(dir), side(side) {}
    virtual ~Base() = default;
    virtual cn_bc_kind kind() const { return CN_BC_BASE; }
    virtual double value() const { return 0.0; }
    virtual std::string name() const { return "Base"; }
    size_t dir, side;
};
struct Dirichlet : Base {
    Dirichlet(size_t dir, size_t side, double v) : Base(dir, side), v(v) {}
    cn_bc_kind kind() const override { return CN_BC_DIRICHLET; }
    double value() const override { return v; }
    std::string name() const override { return "Dirichlet"; }
    double &getValue() { return v; }
    double v;
};
struct Absorbing : Base {
    using Base::Base;
    cn_bc_kind kind() const override { return CN_BC_ABSORBING; }
    std::string name() const override { return "Zeroth-Order Absorbing"; }
};
struct Symmetry : Base {
    Symmetry(size_t dir, size_t side, double sign = 1) : Base(dir, side), sign(sign) {}
    cn_bc_kind kind() const override { return CN_BC_SYMMETRY; }
    double value() const override { return sign; }
    std::string name() const override { return "Symmetry"; }
    double sign;
};
} // namespace BC

namespace Grid {

template <typename T> class Cartesian;

/// The BC vector of one block field: push_back mirrors
/// field.getBC().push_back(new BC::X(...)); the grid keeps the BC objects.
template <typename T> class BCVector {
public:
    BCVector(Cartesian<T> *g, int comp, int block) : g_(g), comp_(comp), block_(block) {}
    void push_back(BC::Base *bc);
    void clear();
    size_t size() const;

private:
    Cartesian<T> *g_;
    int comp_, block_;
};

/// A block field view (component comp of block `flat`).
template <typename T> class BlockField {
public:
    BlockField(Cartesian<T> *g, int flat, int comp) : g_(g), flat_(flat), comp_(comp) {}
    struct State {
        MultiIndex block_index;
    };
    State getState() const;
    Core::IndexRange getIndexRange() const;
    BCVector<T> getBC() { return BCVector<T>(g_, comp_, flat_); }
    int flat() const { return flat_; }
    int comp() const { return comp_; }
    Cartesian<T> &grid() const { return *g_; }

private:
    Cartesian<T> *g_;
    int flat_, comp_;
};

/// Grid::Cartesian(nblocks, block_cells, begin, end) with ncomp components on
/// the GPU.  `entity` as Cubism::EntityType (a FaceContainer grid is three
/// face grids, one per direction): node and face fields have one more entity
/// along a grown dimension in the last block of that dimension.
template <typename T> class Cartesian {
public:
    Cartesian(const MultiIndex &nblocks, const MultiIndex &block_cells,
              const std::array<double, 3> &begin = {0, 0, 0}, const std::array<double, 3> &end = {1, 1, 1},
              int ncomp = 1, cn_entity entity = CN_ENTITY_CELL)
        : nb_(nblocks), n_(block_cells), ncomp_(ncomp), entity_(entity)
    {
        check(cn_grid_create_entity(nblocks.data(), block_cells.data(), ncomp, DType<T>::value, entity, begin.data(),
                                    end.data(), &g_));
        check(cn_grid_layout(g_, &bstride_, &cstride_, nullptr));
    }
    Cartesian(const Cartesian &) = delete;
    Cartesian &operator=(const Cartesian &) = delete;
    ~Cartesian() { cn_grid_destroy(g_); }

    /// Cartesian::operator= (Grid/Cartesian.h:160-169): copy the block data.
    void assign(const Cartesian &c, void *stream = nullptr) { check(cn_grid_copy(g_, c.g_, stream)); }

    size_t size() const { return (size_t)nb_[0] * nb_[1] * nb_[2]; }
    MultiIndex getSize() const { return nb_; }
    MultiIndex getBlockCells() const { return n_; }
    cn_entity getEntity() const { return entity_; }
    int getComponents() const { return ncomp_; }
    /// index-range extent of block field `flat` (Grid/BlockFieldAssembler.h:124-135)
    MultiIndex getBlockExtent(int flat) const
    {
        MultiIndex e = n_;
        const int bi[3] = {flat % nb_[0], (flat / nb_[0]) % nb_[1], flat / (nb_[0] * nb_[1])};
        for (int d = 0; d < 3; ++d)
            if ((entity_ == CN_ENTITY_NODE || entity_ == CN_ENTITY_FACE_X + d) && bi[d] == nb_[d] - 1) ++e[d];
        return e;
    }
    std::array<double, 3> getCellSize() const
    {
        std::array<double, 3> h;
        check(cn_grid_cell_size(g_, h.data()));
        return h;
    }
    int flatIndex(const MultiIndex &p) const { return p[0] + nb_[0] * (p[1] + nb_[1] * p[2]); }
    BlockField<T> operator[](const MultiIndex &p) { return BlockField<T>(this, flatIndex(p), 0); }
    BlockField<T> operator[](size_t i) { return BlockField<T>(this, (int)i, 0); }
    BlockField<T> field(size_t i, int comp) { return BlockField<T>(this, (int)i, comp); }

    int64_t blockStride() const { return bstride_; }
    int64_t componentStride() const { return cstride_; }
    T *deviceData(int comp = 0)
    {
        void *p = nullptr;
        check(cn_grid_data(g_, comp, &p));
        return static_cast<T *>(p);
    }
    /// Host array in the reference SoA order (componentStride() elements).
    void upload(const T *host, int comp = 0, void *stream = nullptr)
    {
        check(cn_grid_upload(g_, comp, host, sizeof(T) * (size_t)cstride_, stream));
    }
    void download(T *host, int comp = 0, void *stream = nullptr) const
    {
        check(cn_grid_download(g_, comp, host, sizeof(T) * (size_t)cstride_, stream));
    }
    void syncBCs(void *stream = nullptr) { check(cn_bc_sync(g_, stream)); }
    cn_grid *raw() { return g_; }
    const cn_grid *raw() const { return g_; }
    std::vector<std::unique_ptr<BC::Base>> &ownedBCs() { return owned_; }

private:
    cn_grid *g_ = nullptr;
    MultiIndex nb_, n_;
    int ncomp_;
    cn_entity entity_;
    int64_t bstride_ = 0, cstride_ = 0;
    std::vector<std::unique_ptr<BC::Base>> owned_;
};

/// Grid::Cartesian<T, Mesh, EntityType::Face, RANK>: every block holds a
/// FaceContainer of three face fields, one per direction, with `ncomp`
/// components each (Block/Field.h:1532-1670), kept as three face grids.
/// field(i, c, d) and getIndexFunctor(c, d) follow the reference's component
/// map (block i, component c, direction d) -> fields[i][d][c]
/// (Block/FieldLabLoader.h:327-364, Grid/Cartesian.h:384-427).
template <typename T> class FaceCartesian {
public:
    FaceCartesian(const MultiIndex &nblocks, const MultiIndex &block_cells,
                  const std::array<double, 3> &begin = {0, 0, 0}, const std::array<double, 3> &end = {1, 1, 1},
                  int ncomp = 1)
        : fx_(nblocks, block_cells, begin, end, ncomp, CN_ENTITY_FACE_X),
          fy_(nblocks, block_cells, begin, end, ncomp, CN_ENTITY_FACE_Y),
          fz_(nblocks, block_cells, begin, end, ncomp, CN_ENTITY_FACE_Z)
    {
    }
    size_t size() const { return fx_.size(); }
    MultiIndex getSize() const { return fx_.getSize(); }
    MultiIndex getBlockCells() const { return fx_.getBlockCells(); }
    std::array<double, 3> getCellSize() const { return fx_.getCellSize(); }
    /// the face grid of direction d (0, 1, 2)
    Cartesian<T> &face(int d)
    {
        if (d < 0 || d > 2) throw std::out_of_range("FaceCartesian: face direction out of range");
        return d == 0 ? fx_ : (d == 1 ? fy_ : fz_);
    }
    BlockField<T> field(size_t i, int c = 0, int d = 0) { return face(d).field(i, c); }
    /// block multi-index -> component c of the face field of direction d
    std::function<BlockField<T>(const MultiIndex &)> getIndexFunctor(int c = 0, int d = 0)
    {
        Cartesian<T> *g = &face(d);
        return [g, c](const MultiIndex &p) { return g->field((size_t)g->flatIndex(p), c); };
    }

private:
    Cartesian<T> fx_, fy_, fz_;
};

template <typename T> void BCVector<T>::push_back(BC::Base *bc)
{
    check(cn_bc_push(g_->raw(), comp_, block_, (int)bc->dir, (int)bc->side, bc->kind(), bc->value()));
    g_->ownedBCs().emplace_back(bc);
}
template <typename T> void BCVector<T>::clear() { check(cn_bc_clear(g_->raw(), comp_, block_)); }
template <typename T> size_t BCVector<T>::size() const
{
    int c = 0;
    check(cn_bc_count(g_->raw(), comp_, block_, &c));
    return (size_t)c;
}

template <typename T> typename BlockField<T>::State BlockField<T>::getState() const
{
    const MultiIndex nb = g_->getSize();
    return State{{flat_ % nb[0], (flat_ / nb[0]) % nb[1], flat_ / (nb[0] * nb[1])}};
}
template <typename T> Core::IndexRange BlockField<T>::getIndexRange() const
{
    Core::IndexRange r;
    r.end = g_->getBlockExtent(flat_);
    return r;
}

} // namespace Grid

namespace Block {
/// Block::FieldLab on the device: a dense (active lab range) device buffer.
template <typename T> class FieldLab {
public:
    FieldLab() = default;
    FieldLab(const FieldLab &) = delete;
    FieldLab &operator=(const FieldLab &) = delete;
    ~FieldLab() { release_(); }

    /// Block/FieldLab.h:104-165: the buffer is (re)allocated for the largest lab
    /// this stencil and range need; a smaller later request reuses it.
    void allocate(const Core::Stencil &s, const Core::IndexRange &max_range, bool force = false)
    {
        s_ = s;
        const MultiIndex e = max_range.getExtent();
        size_t need = 1;
        for (int d = 0; d < 3; ++d) need *= (size_t)(e[d] + 2 - s.getBegin()[d] + s.getEnd()[d] - 1);
        if (force || need > cap_) {
            release_();
            if (cudaMallocWrapper_(need)) throw std::runtime_error("FieldLab: device allocation failed");
            cap_ = need;
        }
        max_ = max_range;
        allocated_ = true;
    }
    bool isAllocated() const { return allocated_; }

    /// Cartesian::loadLab / FieldLab::loadData (Grid/Cartesian.h:412-427,
    /// Block/FieldLab.h:180-224) for block field `f`.
    /// The device buffer holds the grid's largest lab (cn_lab_extent: node and
    /// face grids have one more entity in the last block of a grown dimension);
    /// it grows here if the range given to allocate() was smaller.
    void loadData(Grid::BlockField<T> f, bool apply_bc = true, void *stream = nullptr)
    {
        if (!allocated_) throw std::runtime_error("FieldLab: can not load lab data when not allocated first");
        int ext[3];
        check(cn_lab_extent(f.grid().raw(), s_.raw(), ext));
        const size_t need = (size_t)ext[0] * ext[1] * ext[2];
        if (need > cap_) {
            release_();
            if (cudaMallocWrapper_(need)) throw std::runtime_error("FieldLab: device allocation failed");
            cap_ = need;
        }
        check(cn_lab_fill(f.grid().raw(), f.comp(), s_.raw(), f.flat(), 1, apply_bc ? 1 : 0, buf_, stream));
        field_ = f.flat();
        range_.end = f.getIndexRange().end;
    }
    const Core::Stencil &getActiveStencil() const { return s_; }
    Core::IndexRange getActiveRange() const { return range_; }
    Core::IndexRange getActiveLabRange() const
    {
        Core::IndexRange r;
        r.begin = s_.getBegin();
        for (int d = 0; d < 3; ++d) r.end[d] = range_.end[d] + s_.getEnd()[d] - 1;
        return r;
    }
    int getActiveField() const
    {
        if (field_ < 0) throw std::runtime_error("FieldLab: no field loaded");
        return field_;
    }
    Core::IndexRange getMaximumRange() const { return max_; }
    /// device pointer of the lab (active lab range from getActiveLabRange(),
    /// x fastest, with the strides of the grid's largest lab: cn_lab_extent)
    T *deviceData() { return static_cast<T *>(buf_); }

private:
    Core::Stencil s_;
    Core::IndexRange range_, max_;
    void *buf_ = nullptr;
    size_t cap_ = 0;
    bool allocated_ = false;
    int field_ = -1;
    int cudaMallocWrapper_(size_t n);
    void release_();
};
} // namespace Block

namespace Ops {
template <typename T>
inline void laplacian(Grid::Cartesian<T> &u, Grid::Cartesian<T> &out, int comp = 0, int out_comp = 0,
                      void *stream = nullptr)
{
    check(cn_laplacian(u.raw(), comp, out.raw(), out_comp, stream));
}
template <typename T>
inline void gradient(Grid::Cartesian<T> &u, Grid::Cartesian<T> &out, int comp = 0, int out_comp = 0,
                     void *stream = nullptr)
{
    check(cn_gradient(u.raw(), comp, out.raw(), out_comp, stream));
}
template <typename T>
inline void lapGrad(Grid::Cartesian<T> &u, Grid::Cartesian<T> &lap, Grid::Cartesian<T> &grad, void *stream = nullptr)
{
    check(cn_lap_grad(u.raw(), 0, lap.raw(), 0, grad.raw(), 0, stream));
}
template <typename T>
inline void divergence(Grid::Cartesian<T> &v, Grid::Cartesian<T> &out, void *stream = nullptr)
{
    check(cn_divergence(v.raw(), 0, out.raw(), 0, stream));
}
} // namespace Ops

namespace IO {
/// Global index range of a grid's values: the file range of a whole-grid
/// write (IO/CartesianHDF.h:63-69 with the grid's global mesh).
template <typename T> Core::IndexRange indexRange(const Grid::Cartesian<T> &g)
{
    Core::IndexRange r;
    const cn_entity e = g.getEntity();
    for (int d = 0; d < 3; ++d)
        r.end[d] = g.getSize()[d] * g.getBlockCells()[d] + ((e == CN_ENTITY_NODE || e == CN_ENTITY_FACE_X + d) ? 1 : 0);
    return r;
}

/// Field2AOS over every block (IO/FieldAOS.h:186-194; the block loop of
/// IO/CartesianHDF.h:76-80): d_buf (device, r.size() * ncomp values of
/// FileT) receives components [comp0, comp0 + ncomp) of every point of r
/// inside the grid, interleaved (c + ncomp * flat index, x fastest).
template <typename FileT, typename T>
void Field2AOS(Grid::Cartesian<T> &g, const Core::IndexRange &r, FileT *d_buf, int comp0 = 0, int ncomp = -1,
               void *stream = nullptr)
{
    check(cn_grid_to_aos(g.raw(), comp0, ncomp < 0 ? g.getComponents() - comp0 : ncomp, r.begin.data(),
                         r.end.data(), DType<FileT>::value, d_buf, stream));
}

/// AOS2Field over every block (IO/FieldAOS.h:196-206; IO/CartesianHDF.h:182-186).
template <typename FileT, typename T>
void AOS2Field(const FileT *d_buf, const Core::IndexRange &r, Grid::Cartesian<T> &g, int comp0 = 0, int ncomp = -1,
               void *stream = nullptr)
{
    check(cn_grid_from_aos(g.raw(), comp0, ncomp < 0 ? g.getComponents() - comp0 : ncomp, r.begin.data(),
                           r.end.data(), DType<FileT>::value, d_buf, stream));
}

/// The file buffer of CartesianWriteHDF<FileT> in host memory: gathered on
/// the device, copied down once (synchronous).
template <typename FileT, typename T> std::vector<FileT> gatherAOS(Grid::Cartesian<T> &g, const Core::IndexRange &r)
{
    const size_t n = r.size() * (size_t)g.getComponents();
    std::vector<FileT> host(n);
    void *d = nullptr;
    check(cn_device_alloc(n * sizeof(FileT), &d));
    const cn_status st = cn_grid_to_aos(g.raw(), 0, g.getComponents(), r.begin.data(), r.end.data(),
                                        DType<FileT>::value, d, nullptr);
    const cn_status cp = st == CN_OK ? cn_memcpy(host.data(), d, n * sizeof(FileT), nullptr) : st;
    cn_device_free(d);
    check(st);
    check(cp);
    return host;
}

/// IO::CartesianWriteHDF (IO/CartesianHDF.h:113-131 with
/// src/IO/HDFDriver.cpp:25-111): the whole grid as dataset "data" of dims
/// (z, y, x, components) and type FileT in `fname.h5`, plus the XDMF wrapper
/// `fname.xmf` for cell and node data when create_xdmf.  The HDF5 file is
/// written by the library (no libhdf5 needed).
template <typename FileT, typename T>
void CartesianWriteHDF(const std::string &fname, const std::string &aname, Grid::Cartesian<T> &grid, double time,
                       size_t = 0, bool create_xdmf = true)
{
    const Core::IndexRange r = indexRange(grid);
    check(cn_grid_write_hdf(grid.raw(), fname.c_str(), aname.c_str(), 0, grid.getComponents(), r.begin.data(),
                            r.end.data(), DType<FileT>::value, time, create_xdmf ? 1 : 0, nullptr));
}
/// The face grid of direction face_dir of a face container
/// (IO/FieldAOS.h:136-149); no XDMF wrapper for face data, as in the reference.
template <typename FileT, typename T>
void CartesianWriteHDF(const std::string &fname, const std::string &aname, Grid::FaceCartesian<T> &grid, double time,
                       size_t face_dir = 0, bool create_xdmf = true)
{
    CartesianWriteHDF<FileT>(fname, aname, grid.face((int)face_dir), time, 0, create_xdmf);
}
/// IO::CartesianReadHDF (IO/CartesianHDF.h:206-220 with
/// src/IO/HDFDriver.cpp:113-165): the hyperslab of the grid's extent from
/// `fname.h5`; a missing file throws "CartesianReadHDF: File 'fname' does not
/// exist", as the reference.
template <typename FileT, typename T> void CartesianReadHDF(const std::string &fname, Grid::Cartesian<T> &grid, size_t = 0)
{
    const Core::IndexRange r = indexRange(grid);
    check(cn_grid_read_hdf(grid.raw(), fname.c_str(), 0, grid.getComponents(), r.begin.data(), r.end.data(),
                           DType<FileT>::value, nullptr));
}
template <typename FileT, typename T>
void CartesianReadHDF(const std::string &fname, Grid::FaceCartesian<T> &grid, size_t face_dir = 0)
{
    CartesianReadHDF<FileT>(fname, grid.face((int)face_dir));
}
} // namespace IO

} // namespace cubism_b200

template <typename T> int cubism_b200::Block::FieldLab<T>::cudaMallocWrapper_(size_t n)
{
    return cn_device_alloc(n * sizeof(T), &buf_) == CN_OK ? 0 : 1;
}
template <typename T> void cubism_b200::Block::FieldLab<T>::release_()
{
    if (buf_) cn_device_free(buf_);
    buf_ = nullptr;
    cap_ = 0;
}
