// TEST INFRASTRUCTURE ONLY: host stand-in for the few Thrust pieces the reference's FM and LOD
// headers use.  device_vector is host memory; sort_by_key is a stable sort by signed key (the
// order Thrust's device sort gives: key -1 first), parallel through libstdc++'s OpenMP mode.
#pragma once
#include <parallel/algorithm>

#include <cstring>
#include <numeric>
#include <vector>

namespace thrust {
template <class T>
struct device_vector : std::vector<T> {
    using std::vector<T>::vector;
};
template <class T>
using host_vector = std::vector<T>;
template <class T>
inline T* raw_pointer_cast(T* p) { return p; }

template <class K, class It>
void sort_by_key(K* kb, K* ke, It vb) {
    const long long n = ke - kb;
    std::vector<long long> idx(n);
    std::iota(idx.begin(), idx.end(), 0LL);
    __gnu_parallel::stable_sort(idx.begin(), idx.end(), [kb](long long a, long long b) { return kb[a] < kb[b]; });
    using V = typename std::iterator_traits<It>::value_type;
    std::vector<V> vals(n);
    std::vector<K> keys(n);
    V* v = &*vb;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < n; ++i) {
        vals[i] = v[idx[i]];
        keys[i] = kb[idx[i]];
    }
    std::memcpy(static_cast<void*>(v), vals.data(), sizeof(V) * n);
    std::memcpy(kb, keys.data(), sizeof(K) * n);
}
}  // namespace thrust
