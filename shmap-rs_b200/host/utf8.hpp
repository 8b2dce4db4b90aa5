// Record names as the reference turns header bytes into a String:
// String::from_utf8_lossy (src/io/mod.rs:408-410). Every maximal subpart of an
// ill-formed UTF-8 sequence (a lead byte and the continuation bytes that
// still fit the Unicode well-formed byte table) becomes one U+FFFD
// (EF BF BD); well-formed sequences are copied unchanged.
#pragma once
#include <string>

namespace shm {

inline std::string utf8_lossy(const char* s, size_t n) {
    const unsigned char* p = (const unsigned char*)s;
    std::string out;
    out.reserve(n);
    size_t i = 0;
    while (i < n) {
        const unsigned c = p[i];
        if (c < 0x80) {
            out += (char)c;
            i++;
            continue;
        }
        int need = 0;
        unsigned lo = 0x80, hi = 0xbf;  // the range of the first continuation byte
        if (c >= 0xc2 && c <= 0xdf) need = 1;
        else if (c == 0xe0) need = 2, lo = 0xa0;
        else if ((c >= 0xe1 && c <= 0xec) || c == 0xee || c == 0xef) need = 2;
        else if (c == 0xed) need = 2, hi = 0x9f;
        else if (c == 0xf0) need = 3, lo = 0x90;
        else if (c >= 0xf1 && c <= 0xf3) need = 3;
        else if (c == 0xf4) need = 3, hi = 0x8f;
        size_t j = i + 1;
        int got = 0;
        while (need && got < need && j < n) {
            const unsigned d = p[j];
            if (d < (got ? 0x80u : lo) || d > (got ? 0xbfu : hi)) break;
            j++;
            got++;
        }
        if (need && got == need) out.append(s + i, j - i);
        else out += "\xef\xbf\xbd";
        i = j;
    }
    return out;
}

inline std::string utf8_lossy(const std::string& s) { return utf8_lossy(s.data(), s.size()); }

}  // namespace shm
