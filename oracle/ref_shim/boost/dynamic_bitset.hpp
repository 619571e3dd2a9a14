// Minimal stand-in for boost::dynamic_bitset, used only to compile the reference's own sources
// (its hash tables keep visited/marked flags in one; Boost is not installed in this image).
// It covers exactly the operations the reference calls: construction with a size, operator[]
// read and write, resize(n, value) and reset().  The flags are bookkeeping; no arithmetic of the
// contraction depends on them.  Test infrastructure only: nothing in the product links this.
#ifndef PTC_REF_SHIM_DYNAMIC_BITSET_HPP
#define PTC_REF_SHIM_DYNAMIC_BITSET_HPP

#include <cstddef>
#include <vector>

namespace boost {

template <typename Block = unsigned long, typename Allocator = std::allocator<Block>>
class dynamic_bitset {
  public:
    dynamic_bitset() = default;
    explicit dynamic_bitset(std::size_t n) : bits_(n, false) {}

    std::vector<bool>::reference operator[](std::size_t i) { return bits_[i]; }
    bool operator[](std::size_t i) const { return bits_[i]; }

    void resize(std::size_t n, bool value = false) { bits_.resize(n, value); }
    void reset() { bits_.assign(bits_.size(), false); }
    std::size_t size() const { return bits_.size(); }

  private:
    std::vector<bool> bits_;
};

}  // namespace boost

#endif
