// ephem_driver.cpp - test infrastructure: a command-line driver around the reference's own ephemeris
// compressor and interpolator (src/modules/ephemeris_compressor.cpp, compiled unchanged by oracle/Makefile),
// used only to record golden fixtures for the compressed-ephemeris decoder's tests.
//
//   ephc orbital IN BLOB EVAL
//   ephc rotational IN BLOB EVAL [ORB]   (see rotational() below)
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

// ephc rotational IN BLOB EVAL [ORB]
// IN   : int64 N, double time_span, N x {w[3], x[3], z[3]} raw samples (rotational_state_t), int64 M, M times
// ORB  : optional orbital samples on the same grid (int64 N, double span, N x {r, v}): compressed first,
//        passed to compress_rotational_data (which then also tries the tidally locked form), and its
//        interpolator's state at each evaluation time is handed to set_orbital_state before the rotation
//        is evaluated, as the reader does
// EVAL : int64 level, int64 format, then for each time {w[3], x[3], z[3], r[3], v[3]} (the rotation of the
//        B-spline form as loaded, with the orbital state it was given), then the same after expand()
static int rotational(int argc, char **argv) {
    static_assert(sizeof(rotational_state_t) == 9 * sizeof(double), "rotational_state_t is nine doubles");
    std::vector<uint8_t> in, orb;
    if (!read_all(argv[2], in) || in.size() < 16) return 3;
    const bool has_orb = argc == 6;
    if (has_orb && (!read_all(argv[5], orb) || orb.size() < 16)) return 3;
    int64_t N, M;
    double span;
    std::memcpy(&N, in.data(), 8);
    std::memcpy(&span, in.data() + 8, 8);
    if (N < 2 || in.size() < 16 + (size_t)N * 72 + 8) return 3;
    MFILE mf;
    fwrite(in.data() + 16, sizeof(rotational_state_t), (size_t)N, &mf);
    std::memcpy(&M, in.data() + 16 + (size_t)N * 72, 8);
    if (M < 0 || in.size() < 16 + (size_t)N * 72 + 8 + (size_t)M * 8) return 3;
    std::vector<double> ts((size_t)M);
    std::memcpy(ts.data(), in.data() + 16 + (size_t)N * 72 + 8, (size_t)M * 8);

    MFILE morb;
    std::vector<uint8_t> orb_blob;
    if (has_orb) {
        int64_t No;
        std::memcpy(&No, orb.data(), 8);
        if (No < 2 || orb.size() < 16 + (size_t)No * 48) return 3;
        fwrite(orb.data() + 16, sizeof(orbital_state_t), (size_t)No, &morb);
        if (ephemeris_compressor::compress_orbital_data(morb, span) <= 0) return 5;
        morb.publish();
        orb_blob.assign(morb.data(), morb.data() + morb.size());
    }
    const int64_t level = ephemeris_compressor::compress_rotational_data(mf, span, has_orb ? &morb : nullptr);
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
        MFILE ro(orb_blob.data(), orb_blob.size());
        ephemeris_interpolator io(has_orb ? &ro : nullptr, span);
        for (int pass = 0; pass < 2; ++pass) {
            if (pass == 1) ip.expand();
            for (double t : ts) {
                orbital_state_t os;
                std::memset(&os, 0, sizeof(os));   // (its vectors have no initialising constructor)
                if (has_orb) io(t, &os);
                ip.set_orbital_state(os.r, os.v);
                rotational_state_t s;
                ip(t, &s);
                const double rec[15] = {s.w.x, s.w.y, s.w.z, s.x.x, s.x.y, s.x.z, s.z.x, s.z.y, s.z.z,
                                        os.r.x, os.r.y, os.r.z, os.v.x, os.v.y, os.v.z};
                out.insert(out.end(), rec, rec + 15);
            }
        }
    }
    std::vector<uint8_t> ev(16 + out.size() * 8);
    std::memcpy(ev.data(), &level, 8);
    std::memcpy(ev.data() + 8, &fmt, 8);
    if (!out.empty()) std::memcpy(ev.data() + 16, out.data(), out.size() * 8);
    return write_all(argv[4], ev.data(), ev.size()) ? 0 : 4;
}

int main(int argc, char **argv) {
    static_assert(sizeof(orbital_state_t) == 6 * sizeof(double), "orbital_state_t is six doubles");
    if ((argc == 5 || argc == 6) && std::strcmp(argv[1], "rotational") == 0) return rotational(argc, argv);
    if (argc != 5 || std::strcmp(argv[1], "orbital") != 0) {
        std::fprintf(stderr, "usage: ephc orbital IN BLOB EVAL | ephc rotational IN BLOB EVAL [ORB]\n");
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
