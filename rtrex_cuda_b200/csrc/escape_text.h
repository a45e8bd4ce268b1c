// Line rules of the Escape edge-list format (loadGraph_Escape,
// RTRex_Sequential/GraphIO.cpp:19-74), shared by the host loader (io.cpp) and
// the device parser (escape.cu) so both read a file the same way:
//   * a line starting with '#' is a comment;
//   * a line of blanks only (space, \t, \r, \n, \v, \f) is skipped;
//   * every other line must start with two decimal integers (optional sign,
//     leading blanks); anything after them is ignored.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define ESC_HD __host__ __device__ inline
#else
#define ESC_HD inline
#endif

namespace rtr {

ESC_HD bool esc_is_space(char c)
{
    return c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\v' || c == '\f';
}

// [p, e) holds one line without its '\n'.
ESC_HD bool esc_blank(const char* p, const char* e)
{
    for (; p < e; ++p)
        if (!esc_is_space(*p)) return false;
    return true;
}

// strtoll-like: skips leading blanks (not '\n'), optional sign, decimal digits.
ESC_HD bool esc_parse_i64(const char*& p, const char* e, int64_t* out)
{
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\v' || *p == '\f')) ++p;
    bool neg = false;
    if (p < e && (*p == '-' || *p == '+')) {
        neg = *p == '-';
        ++p;
    }
    if (p >= e || *p < '0' || *p > '9') return false;
    int64_t v = 0;
    while (p < e && *p >= '0' && *p <= '9') v = v * 10 + (*p++ - '0');
    *out = neg ? -v : v;
    return true;
}

// Kind of the line [p, e): 0 skipped (comment or blank), 1 data line parsed
// into (a, b), 2 data line that does not start with two integers.
ESC_HD int esc_line(const char* p, const char* e, int64_t* a, int64_t* b)
{
    if (p < e && *p == '#') return 0;
    if (esc_blank(p, e)) return 0;
    const char* q = p;
    if (!esc_parse_i64(q, e, a) || !esc_parse_i64(q, e, b)) return 2;
    return 1;
}

}  // namespace rtr
