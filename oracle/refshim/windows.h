/*
 * Minimal Win32 stand-in used only to compile the reference HulkEngine CPU
 * sources with g++ on Linux (test infrastructure; never part of the product).
 *
 * The reference's KD-tree / scene / statistics sources include <windows.h>
 * for a handful of MSVC keywords, a timer and a few bitmap types. This header
 * provides exactly those, implemented over POSIX.
 */
#ifndef HK_REFSHIM_WINDOWS_H
#define HK_REFSHIM_WINDOWS_H

#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <time.h>
#include <limits>
#include <cfloat>
#include <cmath>
#include <smmintrin.h>
#include <mm_malloc.h>

#ifndef __forceinline
#define __forceinline inline __attribute__((always_inline))
#endif
#define __declspec(x) __attribute__((x))
#define _CRT_ALIGN(x) __attribute__((aligned(x)))
#define ALIGN16 __attribute__((aligned(16)))

typedef int BOOL;
#ifndef TRUE
#define TRUE 1
#define FALSE 0
#endif
typedef int64_t __int64;
typedef uint64_t UINT64;
typedef uint32_t DWORD;
typedef uint16_t WORD;
typedef int32_t LONG;

typedef union {
    struct { uint32_t LowPart; int32_t HighPart; } u;
    int64_t QuadPart;
} LARGE_INTEGER;

static inline BOOL QueryPerformanceCounter(LARGE_INTEGER *c) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    c->QuadPart = (int64_t)ts.tv_sec * 1000000000LL + ts.tv_nsec;
    return TRUE;
}
static inline BOOL QueryPerformanceFrequency(LARGE_INTEGER *f) {
    f->QuadPart = 1000000000LL;
    return TRUE;
}
static inline int64_t InterlockedIncrement64(volatile int64_t *p) {
    return __sync_add_and_fetch(p, 1);
}
static inline void DebugBreak(void) {}
static inline void OutputDebugStringA(const char *s) { fputs(s, stderr); }

#pragma pack(push, 2)
typedef struct {
    WORD bfType; DWORD bfSize; WORD bfReserved1; WORD bfReserved2; DWORD bfOffBits;
} BITMAPFILEHEADER;
#pragma pack(pop)
typedef struct {
    DWORD biSize; LONG biWidth; LONG biHeight; WORD biPlanes; WORD biBitCount;
    DWORD biCompression; DWORD biSizeImage; LONG biXPelsPerMeter; LONG biYPelsPerMeter;
    DWORD biClrUsed; DWORD biClrImportant;
} BITMAPINFOHEADER;
#define BI_RGB 0

#endif /* HK_REFSHIM_WINDOWS_H */
