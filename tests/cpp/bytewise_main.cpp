// Checks, on the host, the multi-cell forms of the pulling-scheme,
// equivalence-step and sampling kernels against their per-cell forms: the
// byte-parallel helpers against the per-byte rules for every byte value in
// every position, and whole launches (every thread of the grid in turn) of
// set_filler8, eqopt8, fill_parent4, pyramid_fill4, pyr_mean_u16x2 and
// gather4 against set_filler, eqopt, fill_parent, pyramid_fill, pyr_mean_u16
// and gather on random levels.  Prints the mismatch counts; exit status 1 on
// any.

template <class F>
static void launch_1d(uint64_t threads, unsigned block, F f) {
    blockDim = {block, 1, 1};
    for (uint64_t b = 0; b < (threads + block - 1) / block; ++b)
        for (unsigned t = 0; t < block; ++t) {
            blockIdx = {(unsigned)b, 0, 0};
            threadIdx = {t, 0, 0};
            f();
        }
}

template <class F>
static void launch_3d(unsigned gx, unsigned gy, unsigned gz, unsigned block, F f) {
    blockDim = {block, 1, 1};
    for (unsigned z = 0; z < gz; ++z)
        for (unsigned y = 0; y < gy; ++y)
            for (unsigned x = 0; x < gx; ++x)
                for (unsigned t = 0; t < block; ++t) {
                    blockIdx = {x, y, z};
                    threadIdx = {t, 0, 0};
                    f();
                }
}

template <int MODE>
static uint8_t dil_rule(uint8_t s) {
    if (MODE == 0) return s == kEmpty ? kAscendantNeighbour : (s == kSeed ? kPropagate : s);
    return s == kEmpty ? kBoundary : s;
}

static long check_helpers(std::mt19937 &g) {
    long bad = 0;
    for (int pos = 0; pos < 4; ++pos)
        for (int v = 0; v < 256; ++v)
            for (int r = 0; r < 128; ++r) {
                uint32_t w = g();
                w = (w & ~(0xFFu << (8 * pos))) | ((uint32_t)v << (8 * pos));
                const int m = r;  // every m of bytes_in_1_to's range 0..127
                const uint32_t eq = bytes_eq(w, (uint32_t)v * 0x01010101u), rg = bytes_in_1_to(w, m);
                const unsigned n = g() & 15u;
                const uint32_t t0 = dil_target4<0>(w, n), t1 = dil_target4<1>(w, n);
                const unsigned s0 = high_bits4(dil_source4<0>(w)), s1 = high_bits4(dil_source4<1>(w));
                const uint32_t nb = nibble_high_bytes(n);
                for (int j = 0; j < 4; ++j) {
                    const uint8_t b = (uint8_t)(w >> (8 * j));
                    const uint32_t eb = (eq >> (8 * j)) & 0xFFu, rb = (rg >> (8 * j)) & 0xFFu;
                    bad += eb != (b == (uint8_t)v ? 0x80u : 0u);
                    bad += rb != (b >= 1 && b <= m ? 0x80u : 0u);
                    bad += ((nb >> (8 * j)) & 0xFFu) != (((n >> j) & 1u) ? 0x80u : 0u);
                    bad += ((s0 >> j) & 1u) != (unsigned)dil_source<0>(b);
                    bad += ((s1 >> j) & 1u) != (unsigned)dil_source<1>(b);
                    bad += (uint8_t)(t0 >> (8 * j)) != (((n >> j) & 1u) ? dil_rule<0>(b) : b);
                    bad += (uint8_t)(t1 >> (8 * j)) != (((n >> j) & 1u) ? dil_rule<1>(b) : b);
                }
            }
    // dil_bits16 over a 16-byte word: bit e is cell e's source test
    for (int it = 0; it < 100000; ++it) {
        const uint4 v = make_uint4(g(), g(), g(), g());
        const uint32_t vw[4] = {v.x, v.y, v.z, v.w};
        const unsigned p0 = dil_bits16<0>(v), p1 = dil_bits16<1>(v);
        for (int e = 0; e < 16; ++e) {
            const uint8_t b = (uint8_t)(vw[e >> 2] >> (8 * (e & 3)));
            bad += ((p0 >> e) & 1u) != (unsigned)dil_source<0>(b);
            bad += ((p1 >> e) & 1u) != (unsigned)dil_source<1>(b);
        }
    }
    return bad;
}

static long check_pulling(std::mt19937 &g, long &cases) {
    const uint8_t vals[] = {kEmpty, kSeed, kBoundary, kFiller, kUpsamplingSeed, kAscendant, kPropagate,
                            kAscendantNeighbour};
    long bad = 0;
    for (int it = 0; it < 150; ++it) {
        LevelDims dc, dp;
        dc.yn = 8 * (1 + (int)(g() % 40));
        dc.xn = 1 + (int)(g() % 9);
        dc.zn = 1 + (int)(g() % 7);
        dp.yn = dc.yn / 2;
        dp.xn = (dc.xn + 1) / 2;
        dp.zn = (dc.zn + 1) / 2;
        const size_t nc = (size_t)dc.yn * dc.xn * dc.zn, np = (size_t)dp.yn * dp.xn * dp.zn;
        std::vector<uint8_t> C(nc), P(np);
        const unsigned dens = g() % 8;
        for (auto &v : C) v = g() % 8 < dens ? vals[g() % 8] : kEmpty;
        for (auto &v : P) v = g() % 8 < dens ? vals[g() % 8] : kEmpty;
        const unsigned rg8 = (unsigned)std::max((dc.yn / 8 + 127) / 128, 1);
        const unsigned rg4 = (unsigned)std::max((dp.yn / 4 + 127) / 128, 1);
        {
            auto a = C, b = C;
            launch_1d(nc, 256, [&] { set_filler_kernel(P.data(), dp, a.data(), dc); });
            launch_3d(rg8, dc.xn, dc.zn, 128, [&] { set_filler8_kernel(P.data(), dp, b.data(), dc); });
            bad += a != b;
            ++cases;
        }
        for (int mt = 1; mt <= 2; ++mt) {
            auto a = C, b = C;
            launch_1d(nc, 256, [&] { eqopt_kernel(P.data(), dp, a.data(), dc, mt); });
            const unsigned plane8 = (unsigned)(dc.yn / 8) * dc.xn;
            launch_3d((plane8 + 255) / 256, dc.zn, 1, 256, [&] { eqopt8_kernel(P.data(), dp, b.data(), dc, mt); });
            bad += a != b;
            ++cases;
        }
        {
            auto a = P, b = P;
            launch_1d(np, 256, [&] { fill_parent_kernel(C.data(), dc, a.data(), dp); });
            launch_3d(rg4, dp.xn, dp.zn, 128, [&] { fill_parent4_kernel(C.data(), dc, b.data(), dp); });
            bad += a != b;
            ++cases;
        }
    }
    return bad;
}

// One pyramid step from level di down to d = (di.yn / 2, ceil(di.xn / 2),
// ceil(di.zn / 2)), under the vector kernels' launch conditions.
static long check_pyramids(std::mt19937 &g, long &cases) {
    long bad = 0;
    for (int it = 0; it < 200; ++it) {
        LevelDims di, d;
        di.yn = 8 * (1 + (int)(g() % 24));
        di.xn = 1 + (int)(g() % 9);
        di.zn = 1 + (int)(g() % 7);
        d.yn = di.yn / 2;
        d.xn = (di.xn + 1) / 2;
        d.zn = (di.zn + 1) / 2;
        const size_t ni = (size_t)di.yn * di.xn * di.zn, no = (size_t)d.yn * d.xn * d.zn;
        std::vector<uint8_t> lev(ni);
        for (auto &v : lev) v = (uint8_t)(g() % 14);
        const int level = (int)(g() % 14), is_min = (int)(g() % 2);
        std::vector<uint8_t> o1(no), s1(no), o2(no), s2(no);
        launch_1d(no, 256, [&] { pyramid_fill_kernel(lev.data(), di, o1.data(), s1.data(), d, level, is_min); });
        launch_3d((unsigned)std::max((d.yn / 4 + 127) / 128, 1), d.xn, d.zn, 128,
                  [&] { pyramid_fill4_kernel(lev.data(), di, o2.data(), s2.data(), d, level, is_min); });
        bad += o1 != o2 || s1 != s2;
        std::vector<uint16_t> img(ni), m1(no), m2(no);
        for (auto &v : img) v = (uint16_t)g();
        launch_1d(no, 256, [&] { pyr_mean_u16_kernel(img.data(), di, m1.data(), d); });
        launch_3d((unsigned)std::max((d.yn / 2 + 127) / 128, 1), d.xn, d.zn, 128,
                  [&] { pyr_mean_u16x2_kernel(img.data(), di, m2.data(), d); });
        bad += m1 != m2;
        cases += 2;
    }
    return bad;
}

static long check_gather(std::mt19937 &g, long &cases) {
    long bad = 0;
    for (int it = 0; it < 600; ++it) {
        const LevelDims d{1 + (int)(g() % 300), 1 + (int)(g() % 5), 1 + (int)(g() % 4)};
        const uint64_t rows = (uint64_t)d.xn * d.zn;
        const uint64_t lead = g() % 4 + (g() % 2) * 8;  // particles of the levels before this one
        std::vector<uint64_t> xz(rows + 2);
        xz[0] = 0;
        xz[1] = lead;  // the row ends of this level start at row_base = 2
        std::vector<uint16_t> yv(lead);
        std::vector<int> ys(d.yn);
        for (uint64_t r = 0; r < rows; ++r) {
            const int cnt = g() % 5 == 0 ? 0 : (int)(g() % (d.yn + 1));
            for (int y = 0; y < d.yn; ++y) ys[y] = y;
            std::shuffle(ys.begin(), ys.end(), g);
            std::sort(ys.begin(), ys.begin() + cnt);
            for (int k = 0; k < cnt; ++k) yv.push_back((uint16_t)ys[k]);
            xz[r + 2] = yv.size();
        }
        std::vector<uint16_t> im((size_t)d.yn * rows);
        for (auto &v : im) v = (uint16_t)g();
        std::vector<uint16_t> a(yv.size() + 8, 7), b(yv.size() + 8, 7);
        launch_1d(rows * 32, 256, [&] { gather_kernel(im.data(), d, xz.data(), 2, yv.data(), a.data()); });
        launch_1d(rows * 32, 256, [&] { gather4_kernel(im.data(), d, xz.data(), 2, yv.data(), b.data()); });
        bad += a != b;
        ++cases;
    }
    return bad;
}

int main() {
    std::mt19937 g(20261203);
    long cases = 0;
    const long h = check_helpers(g), p = check_pulling(g, cases), m = check_pyramids(g, cases),
               q = check_gather(g, cases);
    std::printf("helpers %ld, launches %ld + pyramids %ld of %ld + gathers %ld mismatched\n", h, p, m, cases, q);
    return (h || p || m || q) ? 1 : 0;
}
