// si_random.hpp -- host-side random streams shared by the engine's seeded
// generators (si_gen.cpp) and the generate_dataset tool: the splitmix64
// finaliser, a splitmix64 stream of uniform doubles, and a Zipf sampler by
// rejection-inversion (Hormann and Derflinger, "Rejection-inversion to
// generate variates from monotone discrete distributions", 1996).
#pragma once

#include <cmath>
#include <cstdint>

namespace si {

inline uint64_t mix64(uint64_t x) {  // splitmix64 finaliser
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

// Uniform double in [0, 1) from a splitmix64 stream.
struct Stream {
    uint64_t state;
    explicit Stream(uint64_t seed) : state(seed) {}
    uint64_t next() {
        state += 0x9e3779b97f4a7c15ull;
        return mix64(state);
    }
    double uniform() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }
};

// Zipf(s) over {1 .. N} by rejection-inversion.  H is an antiderivative of
// h(x) = x^-s; a continuous variate is drawn by inverting H over
// [H(1.5) - 1, H(N + 0.5)], rounded to the nearest integer k, and accepted if
// it falls under h(k) (the test against shortcut_ accepts most draws without
// evaluating H).
class Zipf {
  public:
    Zipf(uint64_t n, double s) : n_(static_cast<double>(n)), s_(s) {
        h_x1_ = H(1.5) - 1.0;
        h_n_ = H(n_ + 0.5);
        shortcut_ = 2.0 - Hinv(H(2.5) - h(2.0));
    }
    uint64_t operator()(Stream& rng) const {
        for (;;) {
            const double u = h_n_ + rng.uniform() * (h_x1_ - h_n_);
            const double x = Hinv(u);
            double k = std::floor(x + 0.5);
            if (k < 1.0) k = 1.0;
            if (k > n_) k = n_;
            if (k - x <= shortcut_ || u >= H(k + 0.5) - h(k)) return static_cast<uint64_t>(k);
        }
    }

  private:
    double h(double x) const { return std::exp(-s_ * std::log(x)); }
    // H(x) = (x^(1-s) - 1) / (1 - s), with its limit log(x) at s = 1
    double H(double x) const {
        const double lx = std::log(x);
        return helper2((1.0 - s_) * lx) * lx;
    }
    double Hinv(double y) const {
        double t = y * (1.0 - s_);
        if (t < -1.0) t = -1.0;  // rounding guard: x >= 0
        return std::exp(helper1(t) * y);
    }
    // helper1(t) = log(1 + t) / t, helper2(t) = (exp(t) - 1) / t, both -> 1 at t = 0
    static double helper1(double t) { return std::fabs(t) > 1e-8 ? std::log1p(t) / t : 1.0 - t / 2.0; }
    static double helper2(double t) { return std::fabs(t) > 1e-8 ? std::expm1(t) / t : 1.0 + t / 2.0; }
    double n_, s_, h_x1_ = 0, h_n_ = 0, shortcut_ = 0;
};

}  // namespace si
