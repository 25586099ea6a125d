/* POSIX stand-in for the few Win32 calls the reference engine makes for its environment
 * banner and file I/O (oracle test infrastructure only). */
#pragma once
#include <unistd.h>
#include <cstdio>
#include <cstdint>
#include <cstring>
typedef unsigned long DWORD;
typedef int BOOL;
struct SYSTEM_INFO { DWORD dwNumberOfProcessors; };
inline void GetSystemInfo(SYSTEM_INFO* s) {
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    const char* e = getenv("TFIM_REF_THREADS");
    if (e && atoi(e) > 0) n = atoi(e);
    s->dwNumberOfProcessors = (DWORD)(n > 0 ? n : 1);
}
enum { RelationProcessorCore = 0 };
struct SYSTEM_LOGICAL_PROCESSOR_INFORMATION { int Relationship; };
inline BOOL GetLogicalProcessorInformation(SYSTEM_LOGICAL_PROCESSOR_INFORMATION*, DWORD* sz) { *sz = 0; return 0; }
inline void __cpuid(int info[4], int) { info[0] = info[1] = info[2] = info[3] = 0; }
inline unsigned long long __popcnt64(unsigned long long x) { return (unsigned long long)__builtin_popcountll(x); }
inline unsigned __popcnt(unsigned x) { return (unsigned)__builtin_popcount(x); }
#define _fseeki64 fseeko
#define _ftelli64 ftello
#ifndef _MSC_VER
#define _MSC_VER 0
#endif
