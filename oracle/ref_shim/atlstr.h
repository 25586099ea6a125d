/* POSIX stand-in for the ATL CString header, written for building the reference engine
 * sources unmodified on Linux (oracle test infrastructure only). */
#pragma once
#include <string>
#include <cstdio>
#include <cstring>
#include <utility>
#ifndef _T
#define _T(x) x
#endif
class CString : public std::string {
public:
    CString() {}
    CString(const char* s) : std::string(s ? s : "") {}
    CString(const std::string& s) : std::string(s) {}
    template <typename... A> void Format(const char* fmt, A... args) {
        char buf[8192];
        std::snprintf(buf, sizeof buf, fmt, conv(args)...);
        assign(buf);
    }
    void Trim() {
        size_t b = find_first_not_of(" \t\r\n");
        size_t e = find_last_not_of(" \t\r\n");
        if (b == npos) { clear(); return; }
        assign(substr(b, e - b + 1));
    }
private:
    static const char* conv(const CString& s) { return s.c_str(); }
    template <typename T> static T conv(T v) { return v; }
};
inline FILE* _tfopen(const CString& p, const char* mode) { return std::fopen(p.c_str(), mode); }
