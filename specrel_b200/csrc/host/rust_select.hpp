// slice::select_nth_unstable_by as Rust's standard library (core::slice::select, the selection of
// Rust 1.81 and later, with the pivot choice of core::slice::sort::shared::pivot and the branchless
// cyclic Lomuto partition of core::slice::sort::unstable::quicksort for elements of at most 96
// bytes) computes it, restated so that the BVH build's median split (bvh4d.rs:410-425) leaves the
// elements in the reference's order: the tree below such a split depends on that order.
//
// After select_nth_unstable(v, len, index, less): no element before `index` is greater than
// v[index], and none after it is less.
#pragma once
#include <cstddef>
#include <utility>

namespace sr_select {

template <class E, class Less>
void insertion_sort_shift_left(E* v, size_t len, size_t offset, Less& less) {
    for (size_t i = offset; i < len; ++i) {
        if (!less(v[i], v[i - 1])) continue;
        E tmp = std::move(v[i]);
        size_t j = i;
        do {
            v[j] = std::move(v[j - 1]);
            --j;
        } while (j > 0 && less(tmp, v[j - 1]));
        v[j] = std::move(tmp);
    }
}

// median3 / median3_rec / choose_pivot (len >= 8).
template <class E, class Less> size_t median3(const E* v, size_t a, size_t b, size_t c, Less& less) {
    const bool x = less(v[a], v[b]), y = less(v[a], v[c]);
    if (x == y) return (less(v[b], v[c]) ^ x) ? c : b;
    return a;
}
template <class E, class Less> size_t median3_rec(const E* v, size_t a, size_t b, size_t c, size_t n, Less& less) {
    if (n * 8 >= 64) {
        const size_t n8 = n / 8;
        a = median3_rec(v, a, a + n8 * 4, a + n8 * 7, n8, less);
        b = median3_rec(v, b, b + n8 * 4, b + n8 * 7, n8, less);
        c = median3_rec(v, c, c + n8 * 4, c + n8 * 7, n8, less);
    }
    return median3(v, a, b, c, less);
}
template <class E, class Less> size_t choose_pivot(const E* v, size_t len, Less& less) {
    const size_t d8 = len / 8;
    const size_t a = 0, b = d8 * 4, c = d8 * 7;
    return len < 64 ? median3(v, a, b, c, less) : median3_rec(v, a, b, c, d8, less);
}

// partition: the pivot to the front, the rest partitioned around it by the cyclic Lomuto scheme
// (each element in turn written to the boundary, the element there moved to the hole it left; the
// first element is held aside and placed last), then the pivot swapped to the boundary. Returns the
// number of elements less than the pivot.
template <class E, class Less> size_t partition(E* v, size_t len, size_t pivot, Less& less) {
    if (len == 0) return 0;
    std::swap(v[0], v[pivot]);
    const E& p = v[0];
    E* a = v + 1;
    const size_t n = len - 1;
    size_t num_lt = 0;
    if (n > 0) {
        E held = std::move(a[0]);
        size_t gap = 0;
        for (size_t r = 1; r < n; ++r) {
            const bool lt = less(a[r], p);
            a[gap] = std::move(a[num_lt]);
            a[num_lt] = std::move(a[r]);
            gap = r;
            num_lt += lt ? 1 : 0;
        }
        const bool lt = less(held, p);
        a[gap] = std::move(a[num_lt]);
        a[num_lt] = std::move(held);
        num_lt += lt ? 1 : 0;
    }
    std::swap(v[0], v[num_lt]);
    return num_lt;
}

template <class E, class Less> size_t min_index(const E* v, size_t len, Less& less) {
    size_t m = 0;
    for (size_t i = 1; i < len; ++i)
        if (less(v[i], v[m])) m = i;
    return m;
}
template <class E, class Less> size_t max_index(const E* v, size_t len, Less& less) {
    size_t m = 0;
    for (size_t i = 1; i < len; ++i)
        if (less(v[m], v[i])) m = i;
    return m;
}

constexpr size_t INSERTION_SORT_THRESHOLD = 16;

template <class E, class Less> size_t median_idx(const E* v, size_t a, size_t b, size_t c, Less& less) {
    if (less(v[c], v[a])) std::swap(a, c);
    if (less(v[c], v[b])) return c;
    if (less(v[b], v[a])) return a;
    return b;
}

template <class E, class Less>
void ninther(E* v, Less& less, size_t a, size_t b, size_t c, size_t d, size_t e, size_t f, size_t g, size_t h, size_t i) {
    b = median_idx(v, a, b, c, less);
    h = median_idx(v, g, h, i, less);
    if (less(v[h], v[b])) std::swap(b, h);
    if (less(v[f], v[d])) std::swap(d, f);
    if (less(v[e], v[d])) {
        // d stays
    } else if (less(v[f], v[e])) {
        d = f;
    } else {
        if (less(v[e], v[b])) std::swap(v[e], v[b]);
        else if (less(v[h], v[e])) std::swap(v[e], v[h]);
        return;
    }
    if (less(v[d], v[b])) d = b;
    else if (less(v[h], v[d])) d = h;
    std::swap(v[d], v[e]);
}

template <class E, class Less> void median_of_medians(E* v, size_t len, Less& less, size_t k);

template <class E, class Less> size_t median_of_ninthers(E* v, size_t len, Less& less) {
    const size_t frac = len <= 1024 ? len / 12 : len <= 128 * 1024 ? len / 64 : len / 1024;
    const size_t pivot = frac / 2;
    const size_t lo = len / 2 - pivot, hi = frac + lo;
    const size_t gap = (len - 9 * frac) / 4;
    size_t a = lo - 4 * frac - gap, b = hi + gap;
    for (size_t i = lo; i < hi; ++i) {
        ninther(v, less, a, i - frac, b, a + 1, i, b + 1, a + 2, i + frac, b + 2);
        a += 3;
        b += 3;
    }
    median_of_medians(v + lo, frac, less, pivot);
    return partition(v, len, lo + pivot, less);
}

template <class E, class Less> void median_of_medians(E* v, size_t len, Less& less, size_t k) {
    for (;;) {
        if (len <= INSERTION_SORT_THRESHOLD) {
            if (len >= 2) insertion_sort_shift_left(v, len, 1, less);
            return;
        }
        if (k == len - 1) {
            std::swap(v[max_index(v, len, less)], v[k]);
            return;
        }
        if (k == 0) {
            std::swap(v[min_index(v, len, less)], v[k]);
            return;
        }
        const size_t p = median_of_ninthers(v, len, less);
        if (p == k) return;
        if (p > k) {
            len = p;
        } else {
            v += p + 1;
            len -= p + 1;
            k -= p + 1;
        }
    }
}

template <class E, class Less> void select_nth_unstable(E* v, size_t len, size_t index, Less less) {
    if (index >= len) return;
    if (index == len - 1) {
        std::swap(v[max_index(v, len, less)], v[index]);
        return;
    }
    if (index == 0) {
        std::swap(v[min_index(v, len, less)], v[index]);
        return;
    }
    // partition_at_index_loop: at most 16 quickselect rounds, then median of medians. A pivot
    // equal to the one that bounded this part from the left is its smallest element: the part is
    // then split into elements equal to it and greater ones.
    const E* ancestor = nullptr;
    int limit = 16;
    auto less_eq = [&less](const E& a, const E& b) { return !less(b, a); };
    while (len > INSERTION_SORT_THRESHOLD) {
        if (limit == 0) {
            median_of_medians(v, len, less, index);
            return;
        }
        --limit;
        const size_t pivot_pos = choose_pivot(v, len, less);
        if (ancestor && !less(*ancestor, v[pivot_pos])) {
            const size_t mid = partition(v, len, pivot_pos, less_eq) + 1;
            if (mid > index) return;
            v += mid;
            len -= mid;
            index -= mid;
            ancestor = nullptr;
            continue;
        }
        const size_t mid = partition(v, len, pivot_pos, less);
        if (mid < index) {
            ancestor = v + mid;
            v += mid + 1;
            len -= mid + 1;
            index -= mid + 1;
        } else if (mid > index) {
            len = mid;
        } else {
            return;
        }
    }
    if (len >= 2) insertion_sort_shift_left(v, len, 1, less);
}

}  // namespace sr_select
