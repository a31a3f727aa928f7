// CPU oracle for the HBP-ISP stereo path: shared helpers.
//
// This is TEST INFRASTRUCTURE. It restates, on the CPU and in plain C++, the
// reference algorithm (TingmanYan/HBP-ISP) so that the B200 engine can be
// checked against it. Only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / reference legs may load it; the product never does.
//
// Build: make -C oracle  ->  oracle/_build/liboracle.so
// Compiled with -ffp-contract=off: every a*b+c is a rounded multiply followed
// by a rounded add, exactly as the engine's kernels (built with -fmad=false)
// evaluate them, so float results agree bit for bit where the operation order
// agrees.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

namespace orc
{

// __float2int_rd as CUDA defines it: floor, NaN -> 0, saturating at the int
// range (PTX cvt.rmi.s32.f32). Used by read_plane_cost (hbp_isp.cu:217).
inline int f2i_rd(float x)
{
    if (x != x)
        return 0;
    if (x >= 2147483648.0f)
        return 2147483647;
    if (x < -2147483648.0f)
        return (-2147483647 - 1);
    return (int)std::floor(x);
}

// BSD LCG, hbp_isp.cu:551-559: (1103515245 * s + 12345) mod 2^31 in uint32.
inline uint32_t lcg(uint32_t s)
{
    return (1103515245u * s + 12345u) % 2147483648u;
}
// hbp_isp.cu:560-569: advances s and returns s / 2^31 * f in float.
inline float lcg_uniform(uint32_t &s, float f)
{
    s = lcg(s);
    return (float)s / 2147483648.0f * f;
}

struct f4
{
    float x, y, z, w;
};

// Float minimum with CUDA's fminf semantics (a NaN operand yields the other).
inline float fmin_cuda(float a, float b) { return std::fmin(a, b); }
inline float fmax_cuda(float a, float b) { return std::fmax(a, b); }

// The 32-slot sum used by every per-node reduction of the engine: values
// v[0..n) are laid out round-robin over 32 slots (slot j accumulates v[j],
// v[j+32], ... sequentially from 0), then the slots are combined by an xor
// butterfly with offsets 16, 8, 4, 2, 1 (slot i += slot i^off).
// xor butterfly over 32 slots (offsets 16, 8, 4, 2, 1; a[i] = a[i] + a[i^off]),
// the value of slot 0.
template <typename R>
inline R butterfly32(const R *slots)
{
    R a[32];
    for (int i = 0; i < 32; ++i)
        a[i] = slots[i];
    for (int off = 16; off >= 1; off >>= 1)
    {
        R b[32];
        for (int i = 0; i < 32; ++i)
            b[i] = a[i] + a[i ^ off];
        std::memcpy(a, b, sizeof(a));
    }
    return a[0];
}

// Last element of the Hillis-Steele inclusive scan of x[0..m) (m <= 32):
// for off = 1, 2, 4, 8, 16: x[r] = x[r - off] + x[r] for r >= off.
template <typename R>
inline R scan_last(const R *x0, int m)
{
    R a[32];
    for (int i = 0; i < m; ++i)
        a[i] = x0[i];
    for (int off = 1; off < 32; off <<= 1)
    {
        R b[32];
        for (int r = 0; r < m; ++r)
            b[r] = r >= off ? a[r - off] + a[r] : a[r];
        std::memcpy(a, b, sizeof(R) * m);
    }
    return a[m - 1];
}


} // namespace orc
