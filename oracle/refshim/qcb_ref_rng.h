// qcb_ref_rng.h -- force-included (g++ -include) into every reference source compiled into the
// reference oracle (oracle/_ref).  TEST INFRASTRUCTURE ONLY.
//
// The reference draws its heatbath uniforms from std::mt19937_64 through
// std::uniform_real_distribution<double>(0, 1) (src/heatbath/heatbath.cpp:10-30).  The CUDA path
// and the restated oracle draw the same uniforms from a counter-based Philox4x32-10 stream per
// link instead.  To run the reference's own hit() on exactly those uniforms, this header makes
// the name std::mt19937_64 denote a replay engine over that Philox stream:
//
//   * <random> is included first, so the standard engine is declared under its real name;
//   * then `mt19937_64` becomes a macro for `qcb_philox_replay_engine`, a type added to
//     namespace std, so every later `std::mt19937_64` in the reference's sources names it.
//
// Each operator() returns one 64-bit word w whose low 11 bits are zero.  libstdc++'s
// uniform_real_distribution<double>(0, 1) on a 64-bit engine computes double(w) / 2^64 (one call
// of generate_canonical<double, 53>) and then (x * (1 - 0)) + 0, so it returns (w >> 11) * 2^-53
// exactly: the same 53-bit uniform the Philox stream yields on the device.  Both words of a
// Philox call are used in order, (out0:out1) then (out2:out3), as in the device stream.
//
// Adding a name to namespace std is outside what the C++ standard defines; libstdc++ accepts it,
// and this build is pinned to g++ with libstdc++ by its Makefile.
#ifndef QCB_REF_RNG_H
#define QCB_REF_RNG_H

#include <cstdint>
#include <random>

namespace qcb_ref {

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), the same constants as the device stream.
inline void philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += W0;
            k1 += W1;
        }
        const uint64_t p0 = (uint64_t)M0 * c0, p1 = (uint64_t)M1 * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

// Stream tag of the heatbath link stream (word 3 of the counter), as on the device.
constexpr uint32_t TAG_HB = 0x48420001u;

// Uniform random bit generator replaying one link's Philox stream: key = seed, counter =
// (call, link, sweep, tag), two 64-bit words per call.
class PhiloxReplayEngine {
public:
    typedef uint64_t result_type;
    static constexpr result_type min() { return 0; }
    static constexpr result_type max() { return ~(result_type)0; }

    PhiloxReplayEngine() : PhiloxReplayEngine(0, 0, 0, TAG_HB) {}
    explicit PhiloxReplayEngine(uint64_t seed) : PhiloxReplayEngine(seed, 0, 0, TAG_HB) {}
    PhiloxReplayEngine(uint64_t seed, uint32_t link, uint32_t sweep, uint32_t tag) {
        key_[0] = (uint32_t)seed;
        key_[1] = (uint32_t)(seed >> 32);
        ctr_[0] = 0;
        ctr_[1] = link;
        ctr_[2] = sweep;
        ctr_[3] = tag;
        have_second_ = false;
        second_ = 0;
        draws_ = 0;
    }
    void seed(uint64_t s) { *this = PhiloxReplayEngine(s); }

    result_type operator()() {
        draws_++;
        if (have_second_) {
            have_second_ = false;
            return second_;
        }
        uint32_t o[4];
        philox4x32_10(ctr_, key_, o);
        ctr_[0]++;
        second_ = word(o[2], o[3]);
        have_second_ = true;
        return word(o[0], o[1]);
    }
    uint64_t draws() const { return draws_; }

private:
    static uint64_t word(uint32_t hi, uint32_t lo) { return ((((uint64_t)hi << 32) | lo) >> 11) << 11; }
    uint32_t key_[2];
    uint32_t ctr_[4];
    uint64_t second_;
    bool have_second_;
    uint64_t draws_;
};

}  // namespace qcb_ref

namespace std {
typedef ::qcb_ref::PhiloxReplayEngine qcb_philox_replay_engine;
}
#define mt19937_64 qcb_philox_replay_engine

#endif
