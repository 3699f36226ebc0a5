// The pseudo-random stream of glibc's rand() (the reference draws its initial
// MPS and its subspace-expansion matrices from it, real_matrix.cc:201-208),
// restated from the published algorithm of glibc's random_r in its default
// TYPE_3 form: an additive lagged-Fibonacci generator over 31 words,
// r[f] += r[b] (mod 2^32) with f - b = 3, output r[f] >> 1; seeded by a
// Park-Miller sequence (16807 * x mod 2^31 - 1, Schrage's decomposition) and
// advanced 310 times before the first output.  Same numbers as srand(seed)
// followed by rand(), without the process-wide lock and state of rand(), so
// each engine owns its stream.
#pragma once

#include <cstdint>

namespace dmrg {

class GlibcRand {
public:
    explicit GlibcRand(unsigned seed = 1) { seed_with(seed); }
    void seed_with(unsigned seed) {
        int32_t word = (int32_t)seed;
        if (word == 0) word = 1;
        r_[0] = (uint32_t)word;
        for (int i = 1; i < kDeg; ++i) {
            const int32_t hi = word / 127773, lo = word % 127773;
            word = 16807 * lo - 2836 * hi;
            if (word < 0) word += 2147483647;
            r_[i] = (uint32_t)word;
        }
        f_ = kSep;
        b_ = 0;
        for (int i = 0; i < 10 * kDeg; ++i) next();
    }
    // The next value of the stream, in [0, 2^31).
    int next() {
        r_[f_] += r_[b_];
        const int v = (int)(r_[f_] >> 1);
        if (++f_ == kDeg) f_ = 0;
        if (++b_ == kDeg) b_ = 0;
        return v;
    }

private:
    static constexpr int kDeg = 31, kSep = 3;
    uint32_t r_[kDeg];
    int f_ = kSep, b_ = 0;
};

}  // namespace dmrg
