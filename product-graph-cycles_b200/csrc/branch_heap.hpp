// branch_heap.hpp -- indexed binary min-heap of the branch-and-bound driver.
//
// Behaviour follows helper/minheap.cpp:16-277 of the reference because the
// pop order of equal values decides which branch is explored next:
//  * push(value, key) is ignored for a key that is present or out of range;
//  * sift-up passes a parent whose value is >= the moving entry's;
//  * sift-down passes to a child whose value is <= the moving entry's,
//    taking the right child when right <= left;
//  * peak() of an empty heap is +infinity; peakKey() of an absent key is -1.
#pragma once
#include <limits>
#include <utility>
#include <vector>

namespace pgc {

class BranchHeap {
  public:
    explicit BranchHeap(long capacity) : item_(capacity, {-1.0, -1}), at_(capacity, -1), cap_(capacity) {}

    bool isEmpty() const { return count_ == 0; }
    long getSize() const { return count_; }
    double peak() const { return count_ == 0 ? std::numeric_limits<double>::infinity() : item_[0].first; }
    double peakKey(long key) const {
        if (key < 0 || key >= cap_ || at_[key] < 0) return -1.0;
        return item_[at_[key]].first;
    }

    void push(double value, long key) {
        if (key < 0 || key >= cap_ || at_[key] >= 0 || count_ == cap_) return;
        const long slot = count_;
        item_[slot] = {value, key};
        at_[key] = slot;
        ++count_;
        up(slot);
    }

    bool decrease(long key, double value) {
        if (key < 0 || key >= cap_) return false;
        const long slot = at_[key];
        if (slot < 0 || !(value < item_[slot].first)) return false;
        item_[slot].first = value;
        up(slot);
        return item_[slot].first != value;
    }

    std::pair<double, long> pop() {
        if (count_ == 0) return {-1.0, -1};
        const std::pair<double, long> top = item_[0];
        const long last = count_ - 1;
        if (last > 0) {
            item_[0] = item_[last];
            at_[item_[0].second] = 0;
        }
        item_[last] = {-1.0, -1};
        at_[top.second] = -1;
        --count_;
        if (count_ > 0) down(0);
        return top;
    }

  private:
    void place(long slot, const std::pair<double, long>& e) {
        item_[slot] = e;
        at_[e.second] = slot;
    }
    void up(long slot) {
        while (slot > 0) {
            const long parent = (slot - 1) / 2;
            if (!(item_[parent].first >= item_[slot].first)) break;
            const auto moving = item_[slot];
            place(slot, item_[parent]);
            place(parent, moving);
            slot = parent;
        }
    }
    void down(long slot) {
        for (;;) {
            const long l = 2 * slot + 1, r = l + 1;
            const bool lOk = l < count_ && item_[l].first <= item_[slot].first;
            const bool rOk = r < count_ && item_[r].first <= item_[slot].first;
            long go = -1;
            if (lOk && rOk) go = (item_[r].first <= item_[l].first) ? r : l;
            else if (lOk) go = l;
            else if (rOk) go = r;
            if (go < 0) return;
            const auto moving = item_[slot];
            place(slot, item_[go]);
            place(go, moving);
            slot = go;
        }
    }

    std::vector<std::pair<double, long>> item_;
    std::vector<long> at_;
    long cap_;
    long count_ = 0;
};

}  // namespace pgc
