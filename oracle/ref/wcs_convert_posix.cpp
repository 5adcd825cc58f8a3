// POSIX replacement for the reference's Win32-only src/utils/wcs_convert.cpp (oracle build only).
// Byte strings are widened/narrowed one byte per character; the reference only uses these
// conversions to open files by name (src/utils/memio.cpp:5-9).
#include <string>

std::wstring strtowcs(std::string str, bool, bool) {
    std::wstring out;
    out.reserve(str.size());
    for (unsigned char c : str) out.push_back((wchar_t)c);
    return out;
}
std::string wcstostr(std::wstring str, bool, bool) {
    std::string out;
    out.reserve(str.size());
    for (wchar_t c : str) out.push_back((char)c);
    return out;
}
