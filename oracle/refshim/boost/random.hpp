// boost/random.hpp stand-in (TEST INFRASTRUCTURE, see qshim.h).  The
// reference draws every random number from one Boost mt19937; the GPU kMC and
// the oracle draw from Philox4x32-10 instead (Salmon et al., SC'11), keyed by
// (random.seed, replica) with a counter per use.  To run the reference's own
// code on the same draws, this stand-in's "mt19937" is a draw source that the
// harness points at the counter each call must use:
//   sequential(purpose): every distribution call takes the next counter
//     {n, 0, purpose, 0}, n = 0, 1, ...   (world set-up)
//   keyed(step, index, purpose): every call consumes the words of the one
//     draw at counter {step, index, purpose, 0} in order   (the step)
// and the distributions map words to values as the GPU and the oracle do:
//   uniform_int [a, b]: a + (w * (b - a + 1)) >> 32, one word
//   uniform_01: ((w_i >> 5) 2^26 + (w_j >> 6)) / 2^53, two words
//   normal: Box-Muller on the four words of a fresh draw.
#pragma once

#include <cmath>
#include <cstdint>
#include <istream>
#include <ostream>
#include <stdexcept>

extern "C" void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

namespace refshim {

struct Draws {
    uint32_t seed = 0, replica = 0;
    bool keyed = false;
    uint32_t step = 0, index = 0, purpose = 0, next = 0;
    uint32_t w[4] = {0, 0, 0, 0};
    int cursor = 4;
    void fetch(uint32_t c0, uint32_t c1, uint32_t c2) {
        const uint32_t ctr[4] = {c0, c1, c2, 0u};
        const uint32_t key[2] = {seed, replica};
        orc_philox4x32_10(ctr, key, w);
        cursor = 0;
    }
    void set_sequential(uint32_t p) {
        keyed = false;
        purpose = p;
        next = 0;
    }
    void set_keyed(uint32_t s, uint32_t i, uint32_t p) {
        keyed = true;
        step = s; index = i; purpose = p;
        fetch(s, i, p);
    }
    // start of one distribution call
    void begin() {
        if (!keyed) fetch(next++, 0u, purpose);
    }
    uint32_t word() {
        if (cursor >= 4) throw std::runtime_error("refshim: a draw's four words are used up");
        return w[cursor++];
    }
};
Draws& draws();

inline double unit_double(uint32_t a, uint32_t b) {
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

}  // namespace refshim

namespace boost {

class mt19937 {
public:
    explicit mt19937(uint32_t seed = 5489u) { this->seed(seed); }
    void seed(uint32_t s) { refshim::draws().seed = s; }
};
inline std::ostream& operator<<(std::ostream& o, const mt19937&) { return o; }
inline std::istream& operator>>(std::istream& i, mt19937&) { return i; }

template <class T = double>
class uniform_01 {
public:
    template <class E>
    T operator()(E&) const {
        refshim::Draws& d = refshim::draws();
        d.begin();
        const uint32_t a = d.word();
        const uint32_t b = d.word();
        return (T)refshim::unit_double(a, b);
    }
};

template <class T = int>
class uniform_int {
public:
    uniform_int(T lo, T hi) : m_lo(lo), m_hi(hi) {}
    template <class E>
    T operator()(E&) const {
        refshim::Draws& d = refshim::draws();
        d.begin();
        const uint64_t n = (uint64_t)((int64_t)m_hi - (int64_t)m_lo + 1);
        return m_lo + (T)(((uint64_t)d.word() * n) >> 32);
    }

private:
    T m_lo, m_hi;
};

template <class T = double>
class uniform_real {
public:
    uniform_real(T lo, T hi) : m_lo(lo), m_hi(hi) {}
    template <class E>
    T operator()(E& e) const {
        return m_lo + (m_hi - m_lo) * uniform_01<T>()(e);
    }

private:
    T m_lo, m_hi;
};

template <class T = double>
class normal_distribution {
public:
    normal_distribution(T mean, T sigma) : m_mean(mean), m_sigma(sigma) {}
    template <class E>
    T operator()(E&) const {
        refshim::Draws& d = refshim::draws();
        d.begin();
        const uint32_t w0 = d.word(), w1 = d.word(), w2 = d.word(), w3 = d.word();
        const double u1 =
            (refshim::unit_double(w0, w1) * 9007199254740991.0 + 1.0) / 9007199254740992.0;
        const double u2 = refshim::unit_double(w2, w3);
        return m_mean + m_sigma * std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
    }

private:
    T m_mean, m_sigma;
};

template <class E, class D>
class variate_generator {
public:
    variate_generator(E e, D d) : m_e(e), m_d(d) {}
    auto operator()() { return m_d(m_e); }

private:
    E m_e;
    D m_d;
};

}  // namespace boost
