// Seeded stand-in for the reference's RandomCluster::fit
// (src/clustering/impl/random_cluster/RandomCluster.cpp:42-136).  TEST
// INFRASTRUCTURE ONLY: linked into the reference IndexGen builds of
// oracle/Makefile (target `host`) in place of RandomCluster.o, so that two
// runs of the reference's clustered loop (src/SparseMat.cpp:927-1095) -- one
// on the CPU path, one on libindexgen_cuda -- see the same clusters.
//
// The reference seeds std::shuffle from std::random_device (its runs never
// repeat) and assigns each candidate to its nearest centre in a python3 GPU
// process (src/gpu_cluster.py).  Here:
//   * centres: call t of fit() (t = 1, 2, ...: one call per iteration of the
//     clustered loop) takes the first actual_k entries of a partial
//     Fisher-Yates shuffle of [0, N) driven by splitmix64 seeded with
//     seed ^ (t * 0xD1B54A32D192ED03), seed from IG_CLUSTER_SEED (default 0)
//     -- the picker of the library's resident clustered solve;
//   * assignment: the oracle's nearest centre (Levenshtein, lowest centre
//     index on ties; pinned to the reference kernel's outputs in
//     tests/golden/assign.npz);
//   * the rest as the reference: k <= 0 gives one cluster, actual_k =
//     min(k, N), clusters keep candidate order, empty clusters are dropped.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <numeric>
#include <string>
#include <vector>

#include "RandomCluster.hpp"
#include "ig_oracle.h"

namespace indexgen {
namespace clustering {
namespace impl {

namespace {

std::atomic<int> g_fit_calls{0};

uint64_t splitmix64(uint64_t &x)
{
    x += 0x9E3779B97F4A7C15ull;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

uint32_t pack_word(const std::string &s)
{
    uint32_t w = 0;
    for (size_t p = 0; p < s.size(); ++p)
        w |= (uint32_t)(s[p] - '0') << (2 * p);
    return w;
}

}  // namespace

RandomCluster::RandomCluster(int k, bool isBinary) : k(k), isBinary(isBinary) {}

std::vector<std::vector<std::string>> RandomCluster::fit(const std::vector<std::string> &data)
{
    if (data.empty())
        return {};
    if (k <= 0)
        return {data};
    const int t = ++g_fit_calls;
    const char *env = std::getenv("IG_CLUSTER_SEED");
    const uint64_t seed = env ? std::strtoull(env, nullptr, 10) : 0;
    const int n = (int)data.size();
    const int actual_k = std::min(k, n);
    std::vector<int> idx((size_t)n);
    std::iota(idx.begin(), idx.end(), 0);
    uint64_t x = seed ^ ((uint64_t)t * 0xD1B54A32D192ED03ull);
    for (int i = 0; i < actual_k; ++i) {
        const int j = i + (int)(splitmix64(x) % (uint64_t)(n - i));
        std::swap(idx[(size_t)i], idx[(size_t)j]);
    }
    const int len = (int)data[0].size();
    std::vector<uint32_t> words((size_t)n), centres((size_t)actual_k);
    for (int i = 0; i < n; ++i)
        words[(size_t)i] = pack_word(data[(size_t)i]);
    for (int c = 0; c < actual_k; ++c)
        centres[(size_t)c] = words[(size_t)idx[(size_t)c]];
    std::vector<int32_t> asg((size_t)n, 0);
    igo_assign_centers(words.data(), n, centres.data(), actual_k, len, 1, asg.data());
    std::vector<std::vector<std::string>> clusters((size_t)actual_k);
    for (int i = 0; i < n; ++i) {
        const int c = asg[(size_t)i];
        clusters[(size_t)(c >= 0 && c < actual_k ? c : 0)].push_back(data[(size_t)i]);
    }
    std::vector<std::vector<std::string>> out;
    for (auto &c : clusters)
        if (!c.empty())
            out.push_back(std::move(c));
    return out;
}

}  // namespace impl
}  // namespace clustering
}  // namespace indexgen
