// TEST INFRASTRUCTURE ONLY — part of the CPU oracle that the parity tests use as the checker.
// Nothing in the shipped library includes, links or calls this file.
//
// The median split of Bvh4D::split (bvh4d.rs:418-424) calls Rust's slice::select_nth_unstable_by,
// whose result order the tree below the split depends on. The reference pins no toolchain; its
// dependencies (wgpu 30) need a recent one, so this restates the selection of Rust 1.81 and later
// (core::slice::select::partition_at_index, with choose_pivot from core::slice::sort::shared::pivot
// and the branchless cyclic Lomuto partition of core::slice::sort::unstable::quicksort, the one
// used for elements of at most 96 bytes). It cannot be run against Rust here (no toolchain), so it
// is held to the selection property and the small-slice insertion sort in the tests.
#pragma once
#include <cstddef>
#include <utility>

namespace orc {
namespace rsel {

// insertion_sort_shift_left(v, 1): each element shifted left past the greater ones before it.
template <class E, class L> void insertion_sort(E* v, size_t n, L& less) {
    for (size_t i = 1; i < n; ++i) {
        if (!less(v[i], v[i - 1])) continue;
        E t = v[i];
        size_t j = i;
        while (true) {
            v[j] = v[j - 1];
            --j;
            if (j == 0 || !less(t, v[j - 1])) break;
        }
        v[j] = t;
    }
}

template <class E, class L> size_t med3(const E* v, size_t a, size_t b, size_t c, L& less) {
    bool x = less(v[a], v[b]), y = less(v[a], v[c]);
    if (x != y) return a;
    return (less(v[b], v[c]) != x) ? c : b;
}

template <class E, class L> size_t med3_rec(const E* v, size_t a, size_t b, size_t c, size_t n, L& less) {
    if (n * 8 >= 64) {  // PSEUDO_MEDIAN_REC_THRESHOLD
        size_t q = n / 8;
        a = med3_rec(v, a, a + 4 * q, a + 7 * q, q, less);
        b = med3_rec(v, b, b + 4 * q, b + 7 * q, q, less);
        c = med3_rec(v, c, c + 4 * q, c + 7 * q, q, less);
    }
    return med3(v, a, b, c, less);
}

template <class E, class L> size_t pick_pivot(const E* v, size_t n, L& less) {
    size_t q = n / 8;
    return n < 64 ? med3(v, 0, 4 * q, 7 * q, less) : med3_rec(v, 0, 4 * q, 7 * q, q, less);
}

// quicksort.rs `partition` with partition_lomuto_branchless_cyclic: returns the count of elements
// less than the pivot, which ends at that index.
template <class E, class L> size_t lomuto(E* v, size_t n, size_t piv, L& less) {
    if (n == 0) return 0;
    std::swap(v[0], v[piv]);
    E* w = v + 1;
    size_t m = n - 1, lt = 0;
    if (m) {
        E first = w[0];
        size_t hole = 0;
        for (size_t k = 1; k < m; ++k) {
            bool is_lt = less(w[k], v[0]);
            w[hole] = w[lt];
            w[lt] = w[k];
            hole = k;
            lt += is_lt;
        }
        bool is_lt = less(first, v[0]);
        w[hole] = w[lt];
        w[lt] = first;
        lt += is_lt;
    }
    std::swap(v[0], v[lt]);
    return lt;
}

template <class E, class L> size_t arg_min(const E* v, size_t n, L& less) {
    size_t m = 0;
    for (size_t i = 1; i < n; ++i) m = less(v[i], v[m]) ? i : m;
    return m;
}
template <class E, class L> size_t arg_max(const E* v, size_t n, L& less) {
    size_t m = 0;
    for (size_t i = 1; i < n; ++i) m = less(v[m], v[i]) ? i : m;
    return m;
}

template <class E, class L> size_t median_idx(const E* v, size_t a, size_t b, size_t c, L& less) {
    if (less(v[c], v[a])) std::swap(a, c);
    if (less(v[c], v[b])) return c;
    if (less(v[b], v[a])) return a;
    return b;
}

template <class E, class L>
void ninther(E* v, L& less, size_t a, size_t b, size_t c, size_t d, size_t e, size_t f, size_t g, size_t h, size_t i) {
    b = median_idx(v, a, b, c, less);
    h = median_idx(v, g, h, i, less);
    if (less(v[h], v[b])) std::swap(b, h);
    if (less(v[f], v[d])) std::swap(d, f);
    if (!less(v[e], v[d])) {
        if (less(v[f], v[e])) {
            d = f;
        } else {
            if (less(v[e], v[b])) std::swap(v[e], v[b]);
            else if (less(v[h], v[e])) std::swap(v[e], v[h]);
            return;
        }
    }
    if (less(v[d], v[b])) d = b;
    else if (less(v[h], v[d])) d = h;
    std::swap(v[d], v[e]);
}

template <class E, class L> void mom(E* v, size_t n, L& less, size_t k);

template <class E, class L> size_t ninthers(E* v, size_t n, L& less) {
    size_t frac = n <= 1024 ? n / 12 : (n <= 131072 ? n / 64 : n / 1024);
    size_t piv = frac / 2, lo = n / 2 - piv, hi = frac + lo, gap = (n - 9 * frac) / 4;
    size_t a = lo - 4 * frac - gap, b = hi + gap;
    for (size_t i = lo; i < hi; ++i, a += 3, b += 3) ninther(v, less, a, i - frac, b, a + 1, i, b + 1, a + 2, i + frac, b + 2);
    mom(v + lo, frac, less, piv);
    return lomuto(v, n, lo + piv, less);
}

// median_of_medians (select.rs): the deterministic fallback after 16 quickselect rounds.
template <class E, class L> void mom(E* v, size_t n, L& less, size_t k) {
    while (true) {
        if (n <= 16) {
            if (n >= 2) insertion_sort(v, n, less);
            return;
        }
        if (k == n - 1) { std::swap(v[arg_max(v, n, less)], v[k]); return; }
        if (k == 0) { std::swap(v[arg_min(v, n, less)], v[k]); return; }
        size_t p = ninthers(v, n, less);
        if (p == k) return;
        if (p > k) { n = p; continue; }
        v += p + 1;
        n -= p + 1;
        k -= p + 1;
    }
}

}  // namespace rsel

// slice::select_nth_unstable_by(index, cmp) with `less` the cmp's Less: partition_at_index.
template <class E, class L> void select_nth_unstable(E* v, size_t n, size_t k, L less) {
    if (k >= n) return;
    if (k == n - 1) { std::swap(v[rsel::arg_max(v, n, less)], v[k]); return; }
    if (k == 0) { std::swap(v[rsel::arg_min(v, n, less)], v[k]); return; }
    auto le = [&less](const E& a, const E& b) { return !less(b, a); };
    const E* ancestor = nullptr;  // the pivot bounding this part from the left, if any
    for (int rounds = 16; n > 16; --rounds) {
        if (rounds == 0) { rsel::mom(v, n, less, k); return; }
        size_t p = rsel::pick_pivot(v, n, less);
        if (ancestor && !less(*ancestor, v[p])) {
            // The pivot equals the smallest: split off the elements equal to it.
            size_t mid = rsel::lomuto(v, n, p, le) + 1;
            if (mid > k) return;
            v += mid;
            n -= mid;
            k -= mid;
            ancestor = nullptr;
            continue;
        }
        size_t mid = rsel::lomuto(v, n, p, less);
        if (mid == k) return;
        if (mid > k) {
            n = mid;
        } else {
            ancestor = v + mid;
            v += mid + 1;
            n -= mid + 1;
            k -= mid + 1;
        }
    }
    if (n >= 2) rsel::insertion_sort(v, n, less);
}

}  // namespace orc
