/*
 * clshim.hpp -- OpenCL C built-ins as plain C++, so that the reference kernel
 * source (src/Simulation/MCLightPropagation.cl, AMD static C++ dialect) can be
 * compiled for the host CPU and run one work-item at a time.
 *
 * TEST INFRASTRUCTURE ONLY: used by oracle/build_ref.py to build oracle/_ref/,
 * the pin for the C restatement in lp_oracle.c.  Nothing in the product uses it.
 *
 * Semantics chosen for the built-ins (and used identically by lp_oracle.c):
 *   dot(a,b)      a.x*b.x + a.y*b.y + a.z*b.z, left to right
 *   normalize(v)  v / sqrt(dot(v,v)); a zero vector is returned unchanged
 *   pown(x,n)     repeated multiplication (x*x for n == 2)
 *   sign(x)       1, -1, +-0 passed through, NaN -> 0
 *   sqrt/log/cos/acos/pow/ceil on float call the C library float functions.
 * Work-items run sequentially, so __local data, atomics and barriers reduce to
 * ordinary memory operations.
 */
#ifndef LP_CLSHIM_HPP
#define LP_CLSHIM_HPP
#include <math.h>
#include <stdint.h>
#include <string.h>

namespace clref {

extern thread_local long g_global_id;
extern long g_global_size;

typedef int event_t;
enum { CLK_LOCAL_MEM_FENCE = 1, CLK_GLOBAL_MEM_FENCE = 2 };
static const float M_PI_F = 3.14159265358979323846f;

struct float2 {
    float x, y;
    float2() : x(0), y(0) {}
    float2(float s) : x(s), y(s) {}
    float2(float a, float b) : x(a), y(b) {}
};
struct float3 {
    float x, y, z;
    float3() : x(0), y(0), z(0) {}
    float3(float s) : x(s), y(s), z(s) {}
    float3(float a, float b, float c) : x(a), y(b), z(c) {}
};
struct f3view {
    float x, y, z;
    operator float3() const { return float3(x, y, z); }
};
struct float4 {
    union {
        struct { float x, y, z, w; };
        f3view xyz;
    };
    float4() : x(0), y(0), z(0), w(0) {}
    float4(float s) : x(s), y(s), z(s), w(s) {}
    float4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    float4(float3 a, float d) : x(a.x), y(a.y), z(a.z), w(d) {}
    float4(float a, float3 b) : x(a), y(b.x), z(b.y), w(b.z) {}
    float4(float2 a, float c, float d) : x(a.x), y(a.y), z(c), w(d) {}
};
struct float8 {
    float s[8];
    float8(float3 a, float3 b, float c, float d)
    {
        s[0] = a.x; s[1] = a.y; s[2] = a.z;
        s[3] = b.x; s[4] = b.y; s[5] = b.z;
        s[6] = c; s[7] = d;
    }
};
struct int2 {
    int x, y;
    int2() : x(0), y(0) {}
    int2(int a, int b) : x(a), y(b) {}
    int2 &operator++() { ++x; ++y; return *this; }
    int2 operator++(int) { int2 t = *this; ++x; ++y; return t; }
};
struct int3 {
    int x, y, z;
    int3() : x(0), y(0), z(0) {}
    int3(int a, int b, int c) : x(a), y(b), z(c) {}
    int3(int2 a, int c) : x(a.x), y(a.y), z(c) {}
};

/* float3 arithmetic (component-wise) */
inline float3 operator+(float3 a, float3 b) { return float3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline float3 operator-(float3 a, float3 b) { return float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float3 operator*(float3 a, float3 b) { return float3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float3 operator/(float3 a, float3 b) { return float3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline float3 operator*(float s, float3 a) { return float3(s * a.x, s * a.y, s * a.z); }
inline float3 operator*(float3 a, float s) { return float3(a.x * s, a.y * s, a.z * s); }
inline float3 operator/(float3 a, float s) { return float3(a.x / s, a.y / s, a.z / s); }
inline float3 operator-(float3 a) { return float3(-a.x, -a.y, -a.z); }
inline float3 &operator+=(float3 &a, float3 b) { a = a + b; return a; }
inline float3 &operator-=(float3 &a, float3 b) { a = a - b; return a; }
inline float3 &operator/=(float3 &a, float s) { a = a / s; return a; }
inline float3 &operator*=(float3 &a, float s) { a = a * s; return a; }
/* float4 arithmetic */
inline float4 operator+(float4 a, float4 b) { return float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
inline float4 operator*(float4 a, float s) { return float4(a.x * s, a.y * s, a.z * s, a.w * s); }
inline float4 operator/(float4 a, float s) { return float4(a.x / s, a.y / s, a.z / s, a.w / s); }

/* math built-ins on float */
inline float sqrt(float x) { return ::sqrtf(x); }
inline float log(float x) { return ::logf(x); }
inline float cos(float x) { return ::cosf(x); }
inline float sin(float x) { return ::sinf(x); }
inline float acos(float x) { return ::acosf(x); }
inline float fabs(float x) { return ::fabsf(x); }
inline float ceil(float x) { return ::ceilf(x); }
inline float pow(float x, float y) { return ::powf(x, y); }
inline float pown(float x, int n)
{
    float r = x;
    for (int i = 1; i < n; ++i) r = r * x;
    return n == 0 ? 1.0f : r;
}
inline float sign(float x)
{
    if (x > 0.0f) return 1.0f;
    if (x < 0.0f) return -1.0f;
    if (x != x) return 0.0f;
    return x;
}
inline float degrees(float r) { return r * (180.0f / M_PI_F); }

/* geometric built-ins */
inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
inline float3 cross(float3 a, float3 b)
{
    return float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float length(float3 v) { return ::sqrtf(dot(v, v)); }
inline float3 normalize(float3 v)
{
    float l = ::sqrtf(dot(v, v));
    if (l == 0.0f) return v;
    return float3(v.x / l, v.y / l, v.z / l);
}
inline float4 normalize(float4 v)
{
    float l = ::sqrtf(dot(v, v));
    if (l == 0.0f) return v;
    return float4(v.x / l, v.y / l, v.z / l, v.w / l);
}

/* vector loads/stores */
inline float2 vload2(long i, const float *p) { return float2(p[2 * i], p[2 * i + 1]); }
inline int2 vload2(long i, const int *p) { return int2(p[2 * i], p[2 * i + 1]); }
inline float3 vload3(long i, const float *p) { return float3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
inline float4 vload4(long i, const float *p)
{
    return float4(p[4 * i], p[4 * i + 1], p[4 * i + 2], p[4 * i + 3]);
}
inline void vstore3(float3 v, long i, float *p) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }
inline void vstore3(int3 v, long i, int *p) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }
inline void vstore4(float4 v, long i, float *p)
{
    p[4 * i] = v.x; p[4 * i + 1] = v.y; p[4 * i + 2] = v.z; p[4 * i + 3] = v.w;
}
inline void vstore8(float8 v, long i, float *p) { memcpy(p + 8 * i, v.s, sizeof v.s); }

/* work-item functions: one work-item per call, one item per work-group */
inline long get_global_id(int) { return g_global_id; }
inline long get_global_size(int) { return g_global_size; }
inline long get_group_id(int) { return g_global_id; }
inline long get_num_groups(int) { return g_global_size; }
inline long get_local_size(int) { return 1; }
template <class T> inline int vec_step(T) { return 1; }

/* synchronisation and atomics reduce to plain memory operations */
inline void barrier(int) {}
inline void mem_fence(int) {}
inline void wait_group_events(int, event_t *) {}
template <class T> inline event_t async_work_group_copy(T *dst, const T *src, long n, event_t e)
{
    memcpy(dst, src, sizeof(T) * (size_t)n);
    return e;
}
inline int atomic_xchg(volatile int *p, int v) { int o = *p; *p = v; return o; }
inline float atomic_xchg(volatile float *p, float v) { float o = *p; *p = v; return o; }
inline unsigned atomic_cmpxchg(volatile unsigned *p, unsigned cmp, unsigned v)
{
    unsigned o = *p;
    if (o == cmp) *p = v;
    return o;
}

} // namespace clref
#endif
