/*
 * Force-included prelude for building the reference's CPU integrator path on Linux
 * (oracle test infrastructure only: never linked into the product library).
 *
 * The reference is an MSVC project. Its hot-path translation units compile under g++ once
 * (1) a few standard headers that MSVC pulls in transitively are included up front, and
 * (2) the Win32 CRT file calls used by src/utils/memio.cpp:5-9,194,205 are mapped to POSIX.
 * Paths are joined with '\\' by the reference loader (src/modules/mass_loader.cpp:111,175,418,427);
 * the _wfopen replacement turns every '\\' into '/'.
 */
#pragma once
#include <atomic>
#include <thread>
#include <cstddef>
#include <cstring>
#include <cstdio>
#include <cstdint>
#include <climits>
#include <cwchar>
#include <string>

static inline FILE *_wfopen(const wchar_t *wname, const wchar_t *wmode) {
    std::string name, mode;
    for (const wchar_t *p = wname; *p; ++p) name.push_back(*p == L'\\' ? '/' : (char)*p);
    for (const wchar_t *p = wmode; *p; ++p) mode.push_back((char)*p);
    return fopen(name.c_str(), mode.c_str());
}
static inline int64_t _ftelli64(FILE *fp) { return (int64_t)ftello(fp); }
static inline int _fseeki64(FILE *fp, int64_t pos, int org) { return fseeko(fp, (off_t)pos, org); }
