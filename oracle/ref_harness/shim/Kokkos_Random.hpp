// Host-only stand-in for Kokkos::Random_XorShift64_Pool (TEST INFRASTRUCTURE, oracle).
//
// The reference seeds one pool per pricing pass and checks a generator state out
// per thread.  Kokkos's own generator source is not available here, so this shim
// uses a documented generator of the same family: xorshift64* (S. Vigna,
// "An experimental exploration of Marsaglia's xorshift generators, scrambled",
// ACM TOMS 42(4), 2016; shifts 12/25/27, multiplier 2685821657736338717), with
// each pool slot seeded through splitmix64 of (seed, slot).  Streams therefore
// differ from a Kokkos build; only the statistics the reference tests pin
// (moments of the normal draws) carry over.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "Kokkos_Core.hpp"

namespace Kokkos {

namespace shim_detail {
inline uint64_t splitmix64(uint64_t &x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
}  // namespace shim_detail

template <class Device = void>
class Random_XorShift64 {
public:
    Random_XorShift64() = default;
    Random_XorShift64(uint64_t state, int slot) : state_(state ? state : 1ULL), slot_(slot) {}

    uint64_t urand64() {
        state_ ^= state_ >> 12;
        state_ ^= state_ << 25;
        state_ ^= state_ >> 27;
        return state_ * 2685821657736338717ULL;
    }
    uint32_t urand() { return static_cast<uint32_t>(urand64() >> 32); }
    // uniform on [0, 1) with 53 (double) / 24 (float) random bits
    double drand() { return static_cast<double>(urand64() >> 11) * (1.0 / 9007199254740992.0); }
    float frand() { return static_cast<float>(urand64() >> 40) * (1.0f / 16777216.0f); }
    double normal() {
        // Marsaglia polar method
        double u, v, s;
        do {
            u = 2.0 * drand() - 1.0;
            v = 2.0 * drand() - 1.0;
            s = u * u + v * v;
        } while (s >= 1.0 || s == 0.0);
        return u * std::sqrt(-2.0 * std::log(s) / s);
    }

    uint64_t state_ = 1;
    int slot_ = 0;
};

template <class Device = void>
class Random_XorShift64_Pool {
public:
    using generator_type = Random_XorShift64<Device>;

    Random_XorShift64_Pool() = default;
    explicit Random_XorShift64_Pool(uint64_t seed) { init(seed, shim_num_threads()); }

    void init(uint64_t seed, int n) {
        states_ = std::make_shared<std::vector<uint64_t>>(static_cast<size_t>(n));
        uint64_t x = seed;
        for (int i = 0; i < n; ++i) {
            uint64_t s = shim_detail::splitmix64(x);
            (*states_)[static_cast<size_t>(i)] = s ? s : 0x9E3779B97F4A7C15ULL;
        }
    }

    generator_type get_state() const {
        const int slot = shim_thread_id();
        return generator_type((*states_)[static_cast<size_t>(slot)], slot);
    }
    void free_state(const generator_type &g) const { (*states_)[static_cast<size_t>(g.slot_)] = g.state_; }

private:
    std::shared_ptr<std::vector<uint64_t>> states_;
};

}  // namespace Kokkos
