// POSIX stand-ins for the Win32 / MSVC runtime names that the reference's
// EDXUtil sources use (Core/Types.h, Core/Memory.h, Windows/Base.h,
// Windows/Timer.h, Math/EDXMath.h, Graphics/ObjMesh.*). Test infrastructure:
// it lets g++ compile those sources unmodified, where they lie, for the
// oracle's reference pins. Nothing here is part of the product.
#pragma once
#include <algorithm>
#include <errno.h>
#include <malloc.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#define __forceinline inline __attribute__((always_inline))

typedef union {
  struct { uint32_t LowPart; int32_t HighPart; };
  long long QuadPart;
} LARGE_INTEGER;

static inline int QueryPerformanceFrequency(LARGE_INTEGER* f) {
  f->QuadPart = 1000000000LL;
  return 1;
}
static inline int QueryPerformanceCounter(LARGE_INTEGER* c) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  c->QuadPart = (long long)t.tv_sec * 1000000000LL + t.tv_nsec;
  return 1;
}
static inline void Sleep(unsigned ms) { usleep(ms * 1000u); }

// _aligned_* on posix_memalign; the size query reports the usable size
static inline void* _aligned_malloc(size_t n, size_t a) {
  void* p = nullptr;
  if (a < sizeof(void*)) a = sizeof(void*);
  return posix_memalign(&p, a, n ? n : 1) ? nullptr : p;
}
static inline void _aligned_free(void* p) { free(p); }
static inline size_t _aligned_msize(void* p, size_t, size_t) { return p ? malloc_usable_size(p) : 0; }
static inline void* _aligned_realloc(void* p, size_t n, size_t a) {
  void* q = _aligned_malloc(n, a);
  if (p && q) {
    const size_t m = malloc_usable_size(p);
    memcpy(q, p, m < n ? m : n);
    free(p);
  }
  return q;
}

// bit scans: index of the highest / lowest set bit; 0 when the mask is 0
static inline unsigned char _BitScanReverse(unsigned long* index, unsigned long mask) {
  if (!mask) return 0;
  *index = (unsigned long)(8 * sizeof(unsigned long) - 1 - __builtin_clzl(mask));
  return 1;
}
static inline unsigned char _BitScanForward(unsigned long* index, unsigned long mask) {
  if (!mask) return 0;
  *index = (unsigned long)__builtin_ctzl(mask);
  return 1;
}

// the bounds-checked CRT calls
static inline int fopen_s(FILE** f, const char* path, const char* mode) {
  *f = fopen(path, mode);
  return *f ? 0 : errno;
}
static inline int strcpy_s(char* dst, size_t size, const char* src) {
  if (!dst || !size) return EINVAL;
  snprintf(dst, size, "%s", src ? src : "");
  return 0;
}
static inline int strncpy_s(char* dst, size_t size, const char* src, size_t count) {
  if (!dst || !size) return EINVAL;
  size_t n = strnlen(src ? src : "", count);
  if (n >= size) n = size - 1;
  memcpy(dst, src, n);
  dst[n] = 0;
  return 0;
}
static inline int strcat_s(char* dst, size_t size, const char* src) {
  if (!dst || !size) return EINVAL;
  const size_t n = strnlen(dst, size);
  if (n < size) snprintf(dst + n, size - n, "%s", src ? src : "");
  return 0;
}
template <size_t N, class... A>
static inline int sprintf_s(char (&buf)[N], const char* fmt, A... a) {
  return snprintf(buf, N, fmt, a...);
}
template <class... A>
static inline int sscanf_s(const char* s, const char* fmt, A... a) {
  return sscanf(s, fmt, a...);
}
template <class... A>
static inline int fscanf_s(FILE* f, const char* fmt, A... a) {
  return fscanf(f, fmt, a...);
}
// "%s" with the buffer's size after it: a width-limited read
static inline int fscanf_s(FILE* f, const char* fmt, char* buf, int size) {
  if (strcmp(fmt, "%s") != 0 || size <= 1) return fscanf(f, fmt, buf);
  char w[32];
  snprintf(w, sizeof w, "%%%ds", size - 1);
  return fscanf(f, w, buf);
}
