/* POSIX stand-ins for the few Win32 calls the reference's CPU sources make
 * (thread start/join and the processor count).  Used only to compile the
 * reference into oracle/_ref/ as a test checker. */
#pragma once
#include <thread>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <limits>
typedef std::thread* HANDLE;
typedef struct { unsigned long dwNumberOfProcessors; } SYSTEM_INFO;
static inline void GetSystemInfo(SYSTEM_INFO* s)
{
    const char* e = getenv("PAGANI_REF_THREADS");
    unsigned long n = e ? strtoul(e, 0, 10) : 0;
    s->dwNumberOfProcessors = n ? n : std::thread::hardware_concurrency();
}
#define INFINITE 0
static inline void WaitForSingleObject(HANDLE h, int) { h->join(); delete h; }
static inline HANDLE _beginthread(void (*fn)(void*), unsigned, void* arg) { return new std::thread(fn, arg); }
static inline char* itoa(int v, char* buf, int) { sprintf(buf, "%d", v); return buf; }
template <size_t L, class... A> static inline int sprintf_s(char (&buf)[L], const char* f, A... a)
{ return snprintf(buf, L, f, a...); }
using std::numeric_limits;
