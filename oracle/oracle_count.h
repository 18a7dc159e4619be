// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle_common.h).
//
// Op-counting f32 for the op-counting build (-DORACLE_COUNT_OPS): the same
// encoder sources, with every f32 arithmetic operation of the reference
// algorithm counted once -- add, sub, mul, div, sqrt, abs, min, max,
// comparisons, int<->float conversions, Rust `as` casts, clamps (two
// comparisons). Integer ALU work and data movement are not counted. The count
// per block is the "algorithmic work" that the BC6H/BC7 roofline divides by.
#pragma once
#include <cmath>
#include <cstdint>

namespace oracle {

extern thread_local uint64_t g_ops;

struct CountedFloat {
    float v;
    CountedFloat() = default;
    constexpr CountedFloat(float x) : v(x) {}
    constexpr CountedFloat(double x) : v((float)x) {}
    CountedFloat(int32_t x) : v((float)x) { g_ops++; }
    CountedFloat(uint32_t x) : v((float)x) { g_ops++; }
    CountedFloat(int64_t x) : v((float)x) { g_ops++; }
    CountedFloat(uint64_t x) : v((float)x) { g_ops++; }
    explicit operator int32_t() const {
        g_ops++;
        return (int32_t)v;
    }
    explicit operator uint32_t() const {
        g_ops++;
        return (uint32_t)v;
    }
    CountedFloat& operator+=(CountedFloat o) { g_ops++; v += o.v; return *this; }
    CountedFloat& operator-=(CountedFloat o) { g_ops++; v -= o.v; return *this; }
    CountedFloat& operator*=(CountedFloat o) { g_ops++; v *= o.v; return *this; }
    CountedFloat& operator/=(CountedFloat o) { g_ops++; v /= o.v; return *this; }
    CountedFloat operator-() const { return CountedFloat(-v); }
};

using real = CountedFloat;

inline real operator+(real a, real b) { g_ops++; return real(a.v + b.v); }
inline real operator-(real a, real b) { g_ops++; return real(a.v - b.v); }
inline real operator*(real a, real b) { g_ops++; return real(a.v * b.v); }
inline real operator/(real a, real b) { g_ops++; return real(a.v / b.v); }
inline bool operator<(real a, real b) { g_ops++; return a.v < b.v; }
inline bool operator>(real a, real b) { g_ops++; return a.v > b.v; }
inline bool operator<=(real a, real b) { g_ops++; return a.v <= b.v; }
inline bool operator>=(real a, real b) { g_ops++; return a.v >= b.v; }
inline bool operator==(real a, real b) { g_ops++; return a.v == b.v; }
inline bool operator!=(real a, real b) { g_ops++; return a.v != b.v; }

inline real sqrt_r(real x) { g_ops++; return real(std::sqrt(x.v)); }
inline real fabs_r(real x) { g_ops++; return real(std::fabs(x.v)); }

// Rust `as i32` / `as u32`: one conversion each.
inline int32_t f2i(float x);
inline uint32_t f2u(float x);
inline int32_t f2i(real x) { g_ops++; return f2i(x.v); }
inline uint32_t f2u(real x) { g_ops++; return f2u(x.v); }
inline real fmin_r(real a, real b) { g_ops++; return real(std::fmin(a.v, b.v)); }
inline real fmax_r(real a, real b) { g_ops++; return real(std::fmax(a.v, b.v)); }
inline real clampf_r(real x, real lo, real hi) {
    g_ops += 2;
    float y = x.v;
    if (y < lo.v) y = lo.v;
    if (y > hi.v) y = hi.v;
    return real(y);
}
inline real sq(real x) { g_ops++; return real(x.v * x.v); }

}  // namespace oracle
