// vsmc_b200/rng.hpp -- host counter-based engines with vSMC's interface.
//
// Drop-in for vsmc::PhiloxEngine<uint32_t,4,10> (include/vsmc/rng/
// philox.hpp:305-524) and vsmc::ThreefryEngine<uint64_t,4,20>
// (include/vsmc/rng/threefry.hpp:263-507): the same (ctr, key) -> words
// function, counter incremented before each block, ctr()/key()/seed()/
// discard(), and std::uniform_random_bit_generator min/max, so the engines
// drive <random> distributions exactly as vSMC's do.  The device kernels
// of libvsmc_cuda produce the same words for the same (key, counter).
#ifndef VSMC_B200_RNG_HPP
#define VSMC_B200_RNG_HPP

#include <array>
#include <cstddef>
#include <cstdint>
#include <istream>
#include <ostream>

namespace vsmc_b200 {

namespace detail {

template <typename T, std::size_t K>
inline void ctr_increment(std::array<T, K> &c)
{
    for (std::size_t i = 0; i != K; ++i)
        if (++c[i] != 0)
            return;
}

template <typename T, std::size_t K>
inline void ctr_add(std::array<T, K> &c, std::uint64_t v)
{
    // little-endian multi-word add; v fits in the first 64 bits
    if (sizeof(T) == 8) {
        std::uint64_t carry = v;
        for (std::size_t i = 0; i != K && carry; ++i) {
            const T s = static_cast<T>(c[i] + carry);
            carry = s < c[i] ? 1 : 0;
            c[i] = s;
        }
    } else {
        std::uint64_t carry = v;
        for (std::size_t i = 0; i != K && carry; ++i) {
            const std::uint64_t s =
                static_cast<std::uint64_t>(c[i]) + (carry & 0xFFFFFFFFull);
            c[i] = static_cast<T>(s);
            carry = (carry >> 32) + (s >> 32);
        }
    }
}

} // namespace detail

/// Philox4x32-10 block function.
inline std::array<std::uint32_t, 4> philox4x32_block(
    std::array<std::uint32_t, 4> c, std::array<std::uint32_t, 2> k)
{
    for (int r = 0; r != 10; ++r) {
        if (r > 0) {
            k[0] += 0x9E3779B9u;
            k[1] += 0xBB67AE85u;
        }
        const std::uint64_t a = 0xCD9E8D57ull * c[2];
        const std::uint64_t b = 0xD2511F53ull * c[0];
        c = {static_cast<std::uint32_t>(a >> 32) ^ k[0] ^ c[1],
             static_cast<std::uint32_t>(a),
             static_cast<std::uint32_t>(b >> 32) ^ k[1] ^ c[3],
             static_cast<std::uint32_t>(b)};
    }
    return c;
}

/// Threefry4x64-20 block function.
inline std::array<std::uint64_t, 4> threefry4x64_block(
    std::array<std::uint64_t, 4> c, const std::array<std::uint64_t, 4> &k)
{
    static const unsigned R0[8] = {14, 52, 23, 5, 25, 46, 58, 32};
    static const unsigned R1[8] = {16, 57, 40, 37, 33, 12, 22, 32};
    std::uint64_t p[5] = {k[0], k[1], k[2], k[3], 0x1BD11BDAA9FC1A22ull};
    for (int i = 0; i != 4; ++i)
        p[4] ^= k[i];
    auto rotl = [](std::uint64_t x, unsigned r) {
        return (x << r) | (x >> (64 - r));
    };
    for (int i = 0; i != 4; ++i)
        c[i] += p[i];
    for (unsigned n = 1; n <= 20; ++n) {
        const unsigned r = (n - 1) % 8;
        if (n % 2) {
            c[0] += c[1];
            c[1] = rotl(c[1], R0[r]) ^ c[0];
            c[2] += c[3];
            c[3] = rotl(c[3], R1[r]) ^ c[2];
        } else {
            c[0] += c[3];
            c[3] = rotl(c[3], R0[r]) ^ c[0];
            c[2] += c[1];
            c[1] = rotl(c[1], R1[r]) ^ c[2];
        }
        if (n % 4 == 0) {
            const unsigned s = n / 4;
            for (unsigned j = 0; j != 4; ++j)
                c[j] += p[(s + j) % 5];
            c[3] += s;
        }
    }
    return c;
}

/// Engine over a block function with vSMC's buffering semantics.
template <typename T, std::size_t KeyWords, typename Derived>
class CounterEngine
{
    public:
    typedef T result_type;
    typedef std::array<T, 4> ctr_type;
    typedef std::array<T, KeyWords> key_type;
    typedef std::array<T, 4> buffer_type;

    explicit CounterEngine(result_type s = 0) { seed(s); }
    explicit CounterEngine(const key_type &k) { seed(k); }

    void seed(result_type s)
    {
        key_.fill(0);
        key_[0] = s;
        ctr_.fill(0);
        index_ = 4;
    }
    void seed(const key_type &k)
    {
        key_ = k;
        ctr_.fill(0);
        index_ = 4;
    }

    ctr_type ctr() const { return ctr_; }
    key_type key() const { return key_; }
    void ctr(const ctr_type &c)
    {
        ctr_ = c;
        index_ = 4;
    }
    void key(const key_type &k)
    {
        key_ = k;
        index_ = 4;
    }

    result_type operator()()
    {
        if (index_ == 4) {
            detail::ctr_increment(ctr_);
            buffer_ = Derived::block(ctr_, key_);
            index_ = 0;
        }
        return buffer_[index_++];
    }

    /// Block for a given counter under the current key.
    buffer_type operator()(const ctr_type &c) const
    {
        return Derived::block(c, key_);
    }

    void discard(std::uint64_t n)
    {
        const std::uint64_t left = 4 - index_;
        if (n <= left) {
            index_ += static_cast<unsigned>(n);
            return;
        }
        n -= left;
        const std::uint64_t blocks = (n - 1) / 4;
        detail::ctr_add(ctr_, blocks);
        index_ = 4;
        operator()();
        index_ = static_cast<unsigned>((n - 1) % 4 + 1);
    }

    /// Words drawn since the counter was zero (valid below 2^64 blocks).
    std::uint64_t words_used() const
    {
        return ctr_[0] == 0 ? 0
                            : (static_cast<std::uint64_t>(ctr_[0]) - 1) * 4 +
                                  index_;
    }

    static constexpr result_type min() { return 0; }
    static constexpr result_type max() { return ~static_cast<result_type>(0); }

    friend bool operator==(const CounterEngine &a, const CounterEngine &b)
    {
        return a.index_ == b.index_ && a.ctr_ == b.ctr_ && a.key_ == b.key_;
    }
    friend bool operator!=(const CounterEngine &a, const CounterEngine &b)
    {
        return !(a == b);
    }

    protected:
    ctr_type ctr_;
    key_type key_;
    buffer_type buffer_;
    unsigned index_ = 4;
};

class Philox4x32
    : public CounterEngine<std::uint32_t, 2, Philox4x32>
{
    public:
    using CounterEngine::CounterEngine;
    static buffer_type block(const ctr_type &c, const key_type &k)
    {
        return philox4x32_block(c, k);
    }
};

class Threefry4x64
    : public CounterEngine<std::uint64_t, 4, Threefry4x64>
{
    public:
    using CounterEngine::CounterEngine;
    static buffer_type block(const ctr_type &c, const key_type &k)
    {
        return threefry4x64_block(c, k);
    }
};

} // namespace vsmc_b200

#endif // VSMC_B200_RNG_HPP
