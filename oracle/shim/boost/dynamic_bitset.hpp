// Minimal stand-in for boost::dynamic_bitset<>, written for this project so
// that the reference's src/boost_bitset.cpp compiles unmodified into
// oracle/_ref/ (Boost is not installed in this image).  It provides the members
// that file uses -- construction with a bit count, set(pos), operator[](pos) --
// with the same semantics: a fixed-size bit vector, all bits initially clear.
//
// Test infrastructure only (oracle build); never part of the product.
#ifndef SI_ORACLE_DYNAMIC_BITSET_SHIM_HPP
#define SI_ORACLE_DYNAMIC_BITSET_SHIM_HPP

#include <cstddef>
#include <cstdint>
#include <memory>
#include <vector>

namespace boost {

template <typename Block = unsigned long, typename Allocator = std::allocator<Block>>
class dynamic_bitset {
public:
    explicit dynamic_bitset(std::size_t num_bits = 0) : words_((num_bits + 63) / 64, 0), bits_(num_bits) {}
    dynamic_bitset& set(std::size_t pos) {
        words_[pos >> 6] |= std::uint64_t(1) << (pos & 63);
        return *this;
    }
    bool operator[](std::size_t pos) const { return (words_[pos >> 6] >> (pos & 63)) & 1u; }
    std::size_t size() const { return bits_; }
    std::size_t count() const {
        std::size_t c = 0;
        for (auto w : words_) c += static_cast<std::size_t>(__builtin_popcountll(w));
        return c;
    }

private:
    std::vector<std::uint64_t> words_;
    std::size_t bits_;
};

}  // namespace boost

#endif
