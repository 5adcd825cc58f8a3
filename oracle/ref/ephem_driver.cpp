// ephem_driver.cpp - test infrastructure: a command-line driver around the reference's own ephemeris
// compressor and interpolator (src/modules/ephemeris_compressor.cpp, compiled unchanged by oracle/Makefile),
// used only to record golden fixtures for the compressed-ephemeris decoder's tests.
//
//   ephc orbital IN BLOB EVAL
//
// IN   : int64 N, double time_span, N x {r[3], v[3]} raw samples (orbital_state_t), int64 M, M times
// BLOB : the compressed record that ephemeris_compressor::compress_orbital_data leaves in the MFILE
//        (empty when the compressor gave up)
// EVAL : int64 level, int64 format, then for each time: {r[3], v[3], GM} of the interpolator's keplerian
//        operator() (GM = its return value), once on the B-spline form as loaded and once after expand()
//        (the Chebyshev form the reader switches to when its memory budget allows)
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "modules/ephemeris_compressor.h"

static bool read_all(const char *path, std::vector<uint8_t> &out) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out.resize(sz > 0 ? (size_t)sz : 0);
    const bool ok = sz <= 0 || std::fread(out.data(), 1, (size_t)sz, f) == (size_t)sz;
    std::fclose(f);
    return ok;
}

static bool write_all(const char *path, const void *p, size_t n) {
    FILE *f = std::fopen(path, "wb");
    if (!f) return false;
    const bool ok = n == 0 || std::fwrite(p, 1, n, f) == n;
    std::fclose(f);
    return ok;
}

int main(int argc, char **argv) {
    static_assert(sizeof(orbital_state_t) == 6 * sizeof(double), "orbital_state_t is six doubles");
    if (argc != 5 || std::strcmp(argv[1], "orbital") != 0) {
        std::fprintf(stderr, "usage: ephc orbital IN BLOB EVAL\n");
        return 2;
    }
    std::vector<uint8_t> in;
    if (!read_all(argv[2], in) || in.size() < 16) return 3;
    const uint8_t *p = in.data();
    int64_t N;
    double span;
    std::memcpy(&N, p, 8);
    std::memcpy(&span, p + 8, 8);
    p += 16;
    if (N < 2 || in.size() < 16 + (size_t)N * 48 + 8) return 3;
    MFILE mf;
    fwrite(p, sizeof(orbital_state_t), (size_t)N, &mf);
    p += (size_t)N * 48;
    int64_t M;
    std::memcpy(&M, p, 8);
    p += 8;
    if (M < 0 || in.size() < 16 + (size_t)N * 48 + 8 + (size_t)M * 8) return 3;
    std::vector<double> ts((size_t)M);
    std::memcpy(ts.data(), p, (size_t)M * 8);

    const int64_t level = ephemeris_compressor::compress_orbital_data(mf, span);
    mf.publish();
    std::vector<uint8_t> blob;
    if (level > 0) blob.assign(mf.data(), mf.data() + mf.size());
    if (!write_all(argv[3], blob.data(), blob.size())) return 4;

    std::vector<double> out;
    int64_t fmt = -1;
    if (level > 0) {
        MFILE rd(blob.data(), blob.size());
        ephemeris_interpolator ip(&rd, span);
        fmt = (int64_t)ip.data_format();
        for (int pass = 0; pass < 2; ++pass) {
            if (pass == 1) ip.expand();
            for (double t : ts) {
                orbital_state_t s;
                keplerian k;
                const double gm = ip(t, &s, k);
                const double rec[7] = {s.r.x, s.r.y, s.r.z, s.v.x, s.v.y, s.v.z, gm};
                out.insert(out.end(), rec, rec + 7);
            }
        }
    }
    std::vector<uint8_t> ev(16 + out.size() * 8);
    std::memcpy(ev.data(), &level, 8);
    std::memcpy(ev.data() + 8, &fmt, 8);
    if (!out.empty()) std::memcpy(ev.data() + 16, out.data(), out.size() * 8);
    return write_all(argv[4], ev.data(), ev.size()) ? 0 : 4;
}
