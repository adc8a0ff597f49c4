// Open-addressing hash map for the host-side tree passes (optimizer,
// topological walk, slot numbering).
//
// Those passes do one lookup per tree node and dominate the time from a
// Tree handle to an uploaded tape; std::unordered_map spends most of that
// time allocating and chasing bucket nodes.  This table keeps keys and
// values inline in one power-of-two array with linear probing, grows at
// half load, and never erases (none of the passes needs it), so a lookup is
// one hash and a short forward scan.
#pragma once
#include <cstddef>
#include <cstdint>
#include <functional>
#include <utility>
#include <vector>

namespace lfb {

/// Multiplicative (Fibonacci) hash of a pointer; low bits of heap pointers
/// are always zero, so the identity hash would cluster.
struct PtrHash {
    size_t operator()(const void* p) const
    {
        return static_cast<size_t>(
            (reinterpret_cast<uintptr_t>(p) >> 3) * 0x9e3779b97f4a7c15ull);
    }
};

template <class K, class V, class Hash, class Eq = std::equal_to<K>>
class FlatMap {
public:
    explicit FlatMap(size_t expected = 16) { reset_table(capacity_for(expected)); }

    size_t size() const { return count_; }

    V* find(const K& k)
    {
        const uint64_t h = mixed(k);
        const uint8_t t = tag_of(h);
        size_t i = slot_of(h);
        while (tags_[i]) {
            if (tags_[i] == t && eq_(slots_[i].first, k)) {
                return &slots_[i].second;
            }
            i = (i + 1) & mask_;
        }
        return nullptr;
    }

    /// Inserts (k, v) unless k is present.  Returns the stored value and
    /// whether this call inserted it.
    template <class VV>
    std::pair<V*, bool> emplace(const K& k, VV&& v)
    {
        if ((count_ + 1) * 2 > slots_.size()) {
            grow();
        }
        const uint64_t h = mixed(k);
        const uint8_t t = tag_of(h);
        size_t i = slot_of(h);
        while (tags_[i]) {
            if (tags_[i] == t && eq_(slots_[i].first, k)) {
                return {&slots_[i].second, false};
            }
            i = (i + 1) & mask_;
        }
        tags_[i] = t;
        slots_[i].first = k;
        slots_[i].second = std::forward<VV>(v);
        ++count_;
        return {&slots_[i].second, true};
    }

    V& operator[](const K& k) { return *emplace(k, V()).first; }

    /// Empties the table, keeping its capacity.
    void clear()
    {
        if (count_ == 0) return;
        for (size_t i = 0; i < slots_.size(); ++i) {
            if (tags_[i]) {
                slots_[i] = std::pair<K, V>();
                tags_[i] = 0;
            }
        }
        count_ = 0;
    }

private:
    static size_t capacity_for(size_t n)
    {
        size_t c = 16;
        while (c < 2 * n) c <<= 1;
        return c;
    }
    void reset_table(size_t cap)
    {
        slots_.assign(cap, std::pair<K, V>());
        tags_.assign(cap, 0);
        mask_ = cap - 1;
        shift_ = 64;
        for (size_t c = cap; c > 1; c >>= 1) --shift_;
        count_ = 0;
    }
    // Fold the hash with a multiply so that weak hashes spread too.
    uint64_t mixed(const K& k) const
    {
        return static_cast<uint64_t>(hash_(k)) * 0x9e3779b97f4a7c15ull;
    }
    // Slot from the high bits, a one-byte tag (never 0) from the low ones:
    // probing reads the dense tag array and touches a slot only on a tag
    // match.
    size_t slot_of(uint64_t h) const
    {
        return static_cast<size_t>(h >> shift_) & mask_;
    }
    static uint8_t tag_of(uint64_t h)
    {
        return static_cast<uint8_t>((h >> 8) | 1);
    }
    void grow()
    {
        std::vector<std::pair<K, V>> old_slots;
        std::vector<uint8_t> old_tags;
        old_slots.swap(slots_);
        old_tags.swap(tags_);
        reset_table(old_slots.size() * 2);
        for (size_t i = 0; i < old_slots.size(); ++i) {
            if (!old_tags[i]) continue;
            const uint64_t h = mixed(old_slots[i].first);
            size_t j = slot_of(h);
            while (tags_[j]) j = (j + 1) & mask_;
            tags_[j] = tag_of(h);
            slots_[j] = std::move(old_slots[i]);
            ++count_;
        }
    }

    std::vector<std::pair<K, V>> slots_;
    std::vector<uint8_t> tags_;
    size_t mask_ = 0;
    unsigned shift_ = 64;
    size_t count_ = 0;
    Hash hash_;
    Eq eq_;
};

}  // namespace lfb
