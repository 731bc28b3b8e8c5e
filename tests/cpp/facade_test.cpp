// The reference's BC, FieldLab and FieldAOS unit-test assertions, through the
// C++ facade on the GPU (test/UnitTests/BC/DirichletTest.cpp, AbsorbingTest.cpp,
// SymmetryTest.cpp, Block/FieldLabTest.cpp:223-291, IO/FieldAOSTest.cpp).
// Exit status 0 = pass.
#include "cubismnova_b200.hpp"

#include <cstdio>
#include <cstdlib>
#include <vector>

using namespace cubism_b200;

static int failures = 0;
#define EXPECT(c)                                                                  \
    do {                                                                           \
        if (!(c)) {                                                                \
            std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #c);             \
            ++failures;                                                            \
        }                                                                          \
    } while (0)

struct HostLab {
    std::vector<int> v;
    int lo, n;
    int E() const { return n + 2 * lo; }
    int operator()(int x, int y, int z) const { return v[(x + lo) + E() * ((y + lo) + E() * (z + lo))]; }
};

static HostLab load(Grid::Cartesian<int> &g, Block::FieldLab<int> &lab)
{
    lab.loadData(g[0]);
    HostLab h;
    h.lo = 3;
    h.n = 16;
    h.v.resize((size_t)h.E() * h.E() * h.E());
    check(cn_memcpy(h.v.data(), lab.deviceData(), sizeof(int) * h.v.size(), nullptr));
    return h;
}

int main()
{
    // FieldAndLab fixture: 16^3 iota int field, stencil (-3,4)
    Grid::Cartesian<int> g({1, 1, 1}, {16, 16, 16});
    std::vector<int> host(g.componentStride());
    for (size_t i = 0; i < host.size(); ++i) host[i] = (int)i;
    g.upload(host.data());
    Block::FieldLab<int> lab;
    try {
        lab.getActiveField();
        EXPECT(false);
    } catch (const std::runtime_error &e) {
        EXPECT(std::string(e.what()) == "FieldLab: no field loaded");
    }
    try {
        lab.loadData(g[0]);
        EXPECT(false);
    } catch (const std::runtime_error &e) {
        EXPECT(std::string(e.what()) == "FieldLab: can not load lab data when not allocated first");
    }
    try {
        Core::Stencil s(1, 4);
        EXPECT(false);
    } catch (const std::runtime_error &e) {
        EXPECT(std::string(e.what()) == "Stencil: begin_ must be <= 0");
    }
    const Core::Stencil s(-3, 4);
    lab.allocate(s, g[0].getIndexRange());
    // Dirichlet on all six faces (DirichletTest.cpp:38-66)
    for (int d = 0; d < 3; ++d)
        for (int side = 0; side < 2; ++side) g[0].getBC().push_back(new BC::Dirichlet(d, side, 10 + 2 * d + side));
    HostLab h = load(g, lab);
    for (int d = 0; d < 3; ++d)
        for (int a = 0; a < 16; ++a)
            for (int b = 0; b < 16; ++b)
                for (int k = 1; k <= 3; ++k) {
                    int lo[3] = {a, b, 0}, hi[3] = {a, b, 0};
                    // the two in-plane coordinates, then the normal one
                    int q0[3], q1[3];
                    for (int m = 0, j = 0; m < 3; ++m) {
                        if (m == d) continue;
                        q0[m] = q1[m] = (j++ == 0) ? a : b;
                    }
                    q0[d] = -k;
                    q1[d] = 15 + k;
                    (void)lo;
                    (void)hi;
                    EXPECT(h(q0[0], q0[1], q0[2]) == 10 + 2 * d);
                    EXPECT(h(q1[0], q1[1], q1[2]) == 11 + 2 * d);
                }
    // Absorbing and Symmetry (AbsorbingTest.cpp, SymmetryTest.cpp)
    g[0].getBC().clear();
    g[0].getBC().push_back(new BC::Absorbing(1, 0));
    g[0].getBC().push_back(new BC::Symmetry(1, 1, -1));
    h = load(g, lab);
    for (int z = 0; z < 16; ++z)
        for (int x = 0; x < 16; ++x)
            for (int k = 1; k <= 3; ++k) {
                EXPECT(h(x, -k, z) == h(x, 0, z));
                EXPECT(h(x, 15 + k, z) == -h(x, 16 - k, z));
            }
    // interior untouched and periodic x ghosts (FieldLabTest.cpp:53-79)
    for (int z = 0; z < 16; ++z)
        for (int y = 0; y < 16; ++y) {
            EXPECT(h(-1, y, z) == h(15, y, z));
            EXPECT(h(16, y, z) == h(0, y, z));
            for (int x = 0; x < 16; ++x) EXPECT(h(x, y, z) == host[x + 16 * (y + 16 * z)]);
        }
    EXPECT(lab.getActiveLabRange().getBegin()[0] == -3 && lab.getActiveLabRange().getEnd()[2] == 19);
    EXPECT(lab.getActiveField() == 0);
    // FaceContainer grid, rank 1 (CartesianTest.cpp:85-103): three face grids;
    // the component map (i, c, d) -> fields[i][d][c] (FieldLabLoader.h:327-364)
    // and the periodic identities of a one-block face lab (FieldLabTest.cpp:
    // 107-114): along its own direction a face field has cells + 1 entities
    {
        Grid::FaceCartesian<int> fg({1, 1, 1}, {4, 4, 4}, {0, 0, 0}, {1, 1, 1}, 2);
        EXPECT(fg.size() == 1);
        Block::FieldLab<int> flab;
        flab.allocate(Core::Stencil(-1, 2), fg.field(0, 0, 0).getIndexRange());
        for (int d = 0; d < 3; ++d) {
            Grid::Cartesian<int> &gd = fg.face(d);
            EXPECT(gd.getEntity() == CN_ENTITY_FACE_X + d);
            const MultiIndex e = gd.getBlockExtent(0);
            for (int k = 0; k < 3; ++k) EXPECT(e[k] == (k == d ? 5 : 4));
            for (int c = 0; c < 2; ++c) {
                std::vector<int> hv(gd.componentStride());
                for (size_t i = 0; i < hv.size(); ++i) hv[i] = (int)(10000 * (d + 1) + 1000 * c + i);
                gd.upload(hv.data(), c);
                Grid::BlockField<int> f = fg.getIndexFunctor(c, d)({0, 0, 0});
                EXPECT(f.comp() == c && &f.grid() == &gd && f.flat() == 0);
                flab.loadData(f);
                const int E0 = e[0] + 2, E1 = e[1] + 2, E2 = e[2] + 2;
                std::vector<int> lv((size_t)E0 * E1 * E2);
                check(cn_memcpy(lv.data(), flab.deviceData(), sizeof(int) * lv.size(), nullptr));
                auto L = [&](int x, int y, int z) { return lv[(x + 1) + E0 * ((y + 1) + E1 * (z + 1))]; };
                auto F = [&](int x, int y, int z) { return hv[x + e[0] * (y + e[1] * z)]; };
                for (int z = 0; z < e[2]; ++z)
                    for (int y = 0; y < e[1]; ++y) {
                        EXPECT(L(-1, y, z) == F(e[0] - 1, y, z));
                        EXPECT(L(e[0], y, z) == F(0, y, z));
                        for (int x = 0; x < e[0]; ++x) EXPECT(L(x, y, z) == F(x, y, z));
                    }
                for (int z = 0; z < e[2]; ++z)
                    for (int x = 0; x < e[0]; ++x) {
                        EXPECT(L(x, -1, z) == F(x, e[1] - 1, z));
                        EXPECT(L(x, e[1], z) == F(x, 0, z));
                    }
                for (int y = 0; y < e[1]; ++y)
                    for (int x = 0; x < e[0]; ++x) {
                        EXPECT(L(x, y, -1) == F(x, y, e[2] - 1));
                        EXPECT(L(x, y, e[2]) == F(x, y, 0));
                    }
            }
        }
        try {
            fg.face(3);
            EXPECT(false);
        } catch (const std::out_of_range &) {
        }
    }
    {
        // IO: the assertions of test/UnitTests/IO/FieldAOSTest.cpp on an 8^3
        // block, then the same over a 2x2x2-block grid (the block loop)
        Grid::Cartesian<float> cf({1, 1, 1}, {8, 8, 8});
        std::vector<float> f(cf.componentStride(), 1.234f);
        cf.upload(f.data());
        const Core::IndexRange all = IO::indexRange(cf);
        std::vector<float> buf = IO::gatherAOS<float>(cf, all);
        EXPECT(buf.size() == 512);
        for (size_t i = 0; i < 512; ++i) EXPECT(buf[i] == f[i]);
        Grid::Cartesian<float> vf({1, 1, 1}, {8, 8, 8}, {0, 0, 0}, {1, 1, 1}, 3);
        for (int c = 0; c < 3; ++c) {
            std::vector<float> v(vf.componentStride(), (c + 1) * 1.234f);
            vf.upload(v.data(), c);
        }
        buf = IO::gatherAOS<float>(vf, all);
        for (size_t i = 0; i < 512; ++i)
            for (int c = 0; c < 3; ++c) EXPECT(buf[c + 3 * i] == (c + 1) * 1.234f);
        // sub-range [2, 5)^3 of a field that is 1.234 there and 0 elsewhere
        Core::IndexRange sub;
        sub.begin = {2, 2, 2};
        sub.end = {5, 5, 5};
        for (int z = 0; z < 8; ++z)
            for (int y = 0; y < 8; ++y)
                for (int x = 0; x < 8; ++x) {
                    const bool in = x >= 2 && x < 5 && y >= 2 && y < 5 && z >= 2 && z < 5;
                    f[x + 8 * (y + 8 * z)] = in ? 1.234f : 0.0f;
                }
        cf.upload(f.data());
        buf = IO::gatherAOS<float>(cf, sub);
        EXPECT(buf.size() == 27);
        for (float v : buf) EXPECT(v == 1.234f);
        // 2x2x2 blocks of 4^3, FP64 grid written as float: the file is the
        // global array, x fastest
        Grid::Cartesian<double> g2({2, 2, 2}, {4, 4, 4});
        std::vector<double> h2(g2.componentStride());
        for (int b = 0; b < 8; ++b)
            for (int i = 0; i < 64; ++i) {
                const int bx = b % 2, by = (b / 2) % 2, bz = b / 4;
                const int x = 4 * bx + i % 4, y = 4 * by + (i / 4) % 4, z = 4 * bz + i / 16;
                h2[(size_t)b * g2.blockStride() + i] = x + 8.0 * (y + 8.0 * z) + 0.5;
            }
        g2.upload(h2.data());
        std::vector<float> b2 = IO::gatherAOS<float>(g2, IO::indexRange(g2));
        for (size_t i = 0; i < b2.size(); ++i) EXPECT(b2[i] == (float)(i + 0.5));
        // read back: AOS2Field of the file into a zeroed grid restores it
        Grid::Cartesian<double> g3({2, 2, 2}, {4, 4, 4});
        std::vector<double> z3(g3.componentStride(), 0.0);
        g3.upload(z3.data());
        void *d = nullptr;
        check(cn_device_alloc(b2.size() * sizeof(float), &d));
        check(cn_memcpy(d, b2.data(), b2.size() * sizeof(float), nullptr));
        IO::AOS2Field(static_cast<const float *>(d), IO::indexRange(g3), g3);
        std::vector<double> back(g3.componentStride());
        g3.download(back.data());
        cn_device_free(d);
        for (int b = 0; b < 8; ++b)
            for (int i = 0; i < 64; ++i)
                EXPECT(back[(size_t)b * g3.blockStride() + i] == h2[(size_t)b * g2.blockStride() + i]);
        // CartesianWriteHDF / CartesianReadHDF through an HDF5 file (FP32
        // file values of an FP64 grid whose values are exact in FP32)
        IO::CartesianWriteHDF<float>("facade_u", "u", g2, 0.5);
        g3.upload(z3.data());
        IO::CartesianReadHDF<float>("facade_u", g3);
        g3.download(back.data());
        for (size_t i = 0; i < back.size(); ++i) EXPECT(back[i] == h2[i]);
        int rank = 0;
        long long dims[32];
        cn_dtype dt;
        check(cn_h5_query("facade_u.h5", "data", &rank, dims, &dt));
        EXPECT(rank == 4 && dims[0] == 8 && dims[1] == 8 && dims[2] == 8 && dims[3] == 1 && dt == CN_FLOAT32);
        try {
            IO::CartesianReadHDF<float>("no_such_file", g3);
            EXPECT(false);
        } catch (const std::runtime_error &e) {
            EXPECT(std::string(e.what()) == "CartesianReadHDF: File 'no_such_file' does not exist");
        }
    }
    std::printf("%s (%d failures)\n", failures ? "FAIL" : "PASS", failures);
    return failures ? 1 : 0;
}
