/*
 * Minimal stand-in for boost::dynamic_bitset, used ONLY to compile the reference's sources
 * for the oracle (test infrastructure).  It provides the subset the reference calls
 * (include/graph_types.h:11-45, src/phase1/seed.cpp:20-190): sized construction, set,
 * operator[], any, count, find_first/find_next, num_blocks, size, clear, resize, |=,
 * boost::move, boost::to_block_range and boost::from_block_range.
 * Bits are stored little-endian in 64-bit blocks, as Boost does.
 */
#ifndef ORACLE_SHIM_BOOST_DYNAMIC_BITSET_HPP
#define ORACLE_SHIM_BOOST_DYNAMIC_BITSET_HPP

#include <cstddef>
#include <cstdint>
#include <utility>
#include <vector>

namespace boost {

template <typename Block = unsigned long>
class dynamic_bitset {
  public:
    typedef Block block_type;
    typedef std::size_t size_type;
    static const size_type npos = static_cast<size_type>(-1);
    static const int bits_per_block = 8 * sizeof(Block);

    dynamic_bitset() : nbits_(0) {}
    explicit dynamic_bitset(size_type n) : nbits_(n), blocks_((n + bits_per_block - 1) / bits_per_block, Block(0)) {}

    size_type size() const { return nbits_; }
    size_type num_blocks() const { return blocks_.size(); }

    void clear() {
        blocks_.clear();
        nbits_ = 0;
    }
    void resize(size_type n, bool value = false) {
        size_type old = nbits_;
        blocks_.resize((n + bits_per_block - 1) / bits_per_block, Block(0));
        nbits_ = n;
        if (value)
            for (size_type i = old; i < n; ++i) set(i);
        trim();
    }
    dynamic_bitset &set(size_type i, bool v = true) {
        if (v)
            blocks_[i / bits_per_block] |= Block(1) << (i % bits_per_block);
        else
            blocks_[i / bits_per_block] &= ~(Block(1) << (i % bits_per_block));
        return *this;
    }
    dynamic_bitset &reset(size_type i) { return set(i, false); }
    bool test(size_type i) const { return (blocks_[i / bits_per_block] >> (i % bits_per_block)) & 1; }
    bool operator[](size_type i) const { return test(i); }

    bool any() const {
        for (Block b : blocks_)
            if (b) return true;
        return false;
    }
    bool none() const { return !any(); }
    size_type count() const {
        size_type c = 0;
        for (Block b : blocks_) c += (size_type)__builtin_popcountl((unsigned long)b);
        return c;
    }
    size_type find_first() const { return find_from(0); }
    size_type find_next(size_type pos) const { return pos + 1 >= nbits_ ? npos : find_from(pos + 1); }

    dynamic_bitset &operator|=(const dynamic_bitset &o) {
        for (size_type i = 0; i < blocks_.size() && i < o.blocks_.size(); ++i) blocks_[i] |= o.blocks_[i];
        return *this;
    }

    std::vector<Block> &blocks() { return blocks_; }
    const std::vector<Block> &blocks() const { return blocks_; }

  private:
    size_type find_from(size_type pos) const {
        size_type bi = pos / bits_per_block;
        if (bi >= blocks_.size()) return npos;
        Block b = blocks_[bi] & (~Block(0) << (pos % bits_per_block));
        while (true) {
            if (b) {
                size_type r = bi * bits_per_block + (size_type)__builtin_ctzl((unsigned long)b);
                return r < nbits_ ? r : npos;
            }
            if (++bi >= blocks_.size()) return npos;
            b = blocks_[bi];
        }
    }
    void trim() {
        size_type extra = nbits_ % bits_per_block;
        if (extra && !blocks_.empty()) blocks_.back() &= (Block(1) << extra) - 1;
    }

    size_type nbits_;
    std::vector<Block> blocks_;
};

template <typename B>
const typename dynamic_bitset<B>::size_type dynamic_bitset<B>::npos;

template <typename B, typename OutIt>
void to_block_range(const dynamic_bitset<B> &b, OutIt out) {
    for (B blk : b.blocks()) *out++ = blk;
}

template <typename InIt, typename B>
void from_block_range(InIt first, InIt last, dynamic_bitset<B> &b) {
    std::size_t i = 0;
    for (; first != last && i < b.blocks().size(); ++first, ++i) b.blocks()[i] = *first;
}

template <typename T>
typename std::remove_reference<T>::type &&move(T &&t) {
    return static_cast<typename std::remove_reference<T>::type &&>(t);
}

}  // namespace boost

#endif
