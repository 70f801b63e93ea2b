// Iteration order of robin_hood::unordered_set<int> / unordered_map<int, T>
// (robin-hood-hashing v3.11.5 by Martin Ankerl, MIT licence, vendored by
// InstantGR as src/robin_hood.h), restated from its published algorithm so that
// the host code here can walk integer keys in the order InstantGR's pin
// selection walks them (src/database.hpp:99-224, 225-242).  Only the keys and
// their slots are modelled; values never change the order.
//
// The table is a power-of-two array of slots plus an overflow buffer of
// min(0.8 * buckets, 255) slots, with one info byte per slot: 0 = empty,
// otherwise (distance from the home slot + 1) * inc + a few hash bits.  For a
// key k:
//   h = murmur3-style mix of (uint64)k: h ^= h >> 33; h *= 0xff51afd7ed558ccd;
//       h ^= h >> 33; then h *= multiplier; h ^= h >> 33
//   info = inc + ((h & 31) >> info_shift), home slot = (h >> 5) & mask
// Insertion walks from the home slot past entries whose info is larger (or
// equal), and places the key there, shifting the following entries up by one
// slot to the next empty one (their info grows by inc).  The table holds at
// most 80% of its buckets; when full it tries to halve inc (one hash bit less
// in the info bytes), otherwise it doubles the buckets and re-inserts the old
// slots in slot order (or, with fewer than 40% used, re-inserts at the same
// size with the next multiplier).  Iteration visits the occupied slots in
// increasing slot order.  clear() empties the slots and resets inc and the
// info shift, and keeps the size, the multiplier and the element limit;
// reset() gives a new, empty table.
#pragma once
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

namespace igr {

class RobinOrder {
public:
    RobinOrder() { reset_empty(); }

    // inserts k if absent; returns true when it was inserted
    bool insert(int k) {
        for (int attempt = 0; attempt < 256; ++attempt) {
            size_t idx;
            uint32_t info;
            key_to_idx(k, idx, info);
            while (info < info_at(idx)) next(info, idx);
            while (info == info_at(idx)) {
                if (keys_[idx] == k) return false;
                next(info, idx);
            }
            if (num_ >= max_allowed_) {
                increase_size();
                continue;
            }
            place(k, idx, info);
            return true;
        }
        return false;  // the table gave up (robin_hood throws overflow_error here)
    }

    bool contains(int k) const {
        if (mask_ == 0) return false;
        size_t idx;
        uint32_t info;
        key_to_idx(k, idx, info);
        while (true) {
            if (info == info_[idx] && keys_[idx] == k) return true;
            next(info, idx);
            if (info > info_[idx]) return false;
        }
    }

    // a freshly constructed table (what a container declared anew gives)
    void reset() {
        reset_empty();
        mult_ = kFirstMultiplier;
    }

    void clear() {
        if (num_ == 0) return;
        std::fill(info_.begin(), info_.end(), 0);
        info_[slots_with_buffer()] = 1;
        num_ = 0;
        inc_ = kInitialInc;
        shift_ = 0;
    }

    size_t size() const { return num_; }

    // keys in iteration order
    template <class F>
    void for_each(F &&f) const {
        if (num_ == 0) return;
        const size_t n = slots_with_buffer();
        for (size_t i = 0; i < n; i++)
            if (info_[i]) f(keys_[i]);
    }

private:
    static constexpr uint32_t kInitialInc = 32;  // 1 << 5 hash bits
    static constexpr uint64_t kMaskInfo = 31;
    static constexpr size_t kInitialBuckets = 8;
    static constexpr uint64_t kFirstMultiplier = 0xc4ceb9fe1a85ec53ULL;
    static constexpr uint64_t kMultiplierStep = 0xc4ceb9fe1a85ec54ULL;

    std::vector<int> keys_;
    std::vector<uint8_t> info_;
    std::vector<int> old_keys_;     // the slots being re-inserted by rehash (storage reused)
    std::vector<uint8_t> old_info_;
    size_t num_ = 0, mask_ = 0, max_allowed_ = 0;
    uint32_t inc_ = kInitialInc, shift_ = 0;
    uint64_t mult_ = kFirstMultiplier;

    static size_t max_allowed(size_t buckets) { return buckets * 80 / 100; }
    static size_t with_buffer(size_t buckets) { return buckets + std::min<size_t>(max_allowed(buckets), 0xFF); }
    size_t slots_with_buffer() const { return with_buffer(mask_ + 1); }

    // the empty table reads one zero info byte at slot 0
    uint32_t info_at(size_t idx) const { return mask_ == 0 ? 0u : info_[idx]; }

    void reset_empty() {
        keys_.assign(1, 0);
        info_.assign(8, 0);
        num_ = mask_ = max_allowed_ = 0;
        inc_ = kInitialInc;
        shift_ = 0;
    }

    void key_to_idx(int k, size_t &idx, uint32_t &info) const {
        uint64_t h = (uint64_t)(int64_t)k;
        h ^= h >> 33;
        h *= 0xff51afd7ed558ccdULL;
        h ^= h >> 33;
        h *= mult_;
        h ^= h >> 33;
        info = inc_ + (uint32_t)((h & kMaskInfo) >> shift_);
        idx = (size_t)(h >> 5) & mask_;
    }

    void next(uint32_t &info, size_t &idx) const {
        idx += 1;
        info += inc_;
    }

    // places a new key at the walk's position idx (info), shifting the run up
    void place(int k, size_t idx, uint32_t info) {
        const size_t at = idx;
        const uint32_t at_info = info;
        if (at_info + inc_ > 0xFF) max_allowed_ = 0;
        while (info_[idx] != 0) next(info, idx);
        if (idx != at) {
            for (size_t i = idx; i != at; --i) keys_[i] = keys_[i - 1];
            for (size_t i = idx; i != at; --i) {
                info_[i] = (uint8_t)(info_[i - 1] + inc_);
                if (info_[i] + inc_ > 0xFF) max_allowed_ = 0;
            }
        }
        keys_[at] = k;
        info_[at] = (uint8_t)at_info;
        ++num_;
    }

    void init_data(size_t buckets) {
        num_ = 0;
        mask_ = buckets - 1;
        max_allowed_ = max_allowed(buckets);
        const size_t n = with_buffer(buckets);
        keys_.assign(n, 0);
        info_.assign(n + 8, 0);
        info_[n] = 1;  // sentinel
        inc_ = kInitialInc;
        shift_ = 0;
    }

    bool try_increase_info() {
        if (inc_ <= 2) return false;
        inc_ >>= 1;
        ++shift_;
        const size_t n = slots_with_buffer();
        // every byte of the info array shifted right by one, eight at a time
        for (size_t i = 0; i < n; i += 8)
            for (size_t j = i; j < i + 8 && j < info_.size(); j++) info_[j] = (uint8_t)(info_[j] >> 1);
        info_[n] = 1;
        max_allowed_ = max_allowed(mask_ + 1);
        return true;
    }

    // re-insertion of a key known to be absent (the rehash path)
    void insert_known_new(int k) {
        if (max_allowed_ == 0 && !try_increase_info()) return;  // robin_hood throws here
        size_t idx;
        uint32_t info;
        key_to_idx(k, idx, info);
        while (info <= info_[idx]) {
            idx += 1;
            info += inc_;
        }
        place(k, idx, info);
    }

    void rehash(size_t buckets) {
        const size_t old_n = with_buffer(mask_ + 1);
        const bool had = mask_ != 0;
        old_keys_.swap(keys_);
        old_info_.swap(info_);
        init_data(buckets);
        if (had && old_n > 1)
            for (size_t i = 0; i < old_n; i++)
                if (old_info_[i] != 0) insert_known_new(old_keys_[i]);
    }

    void increase_size() {
        if (mask_ == 0) {
            init_data(kInitialBuckets);
            return;
        }
        const size_t lim = max_allowed(mask_ + 1);
        if (num_ < lim && try_increase_info()) return;
        if (num_ * 2 < lim) {
            mult_ += kMultiplierStep;
            rehash(mask_ + 1);
        } else {
            rehash((mask_ + 1) * 2);
        }
    }
};

}  // namespace igr
