// FillAdjListGPU on libindexgen_cuda: the body that takes the place of the
// reference's definition in src/SparseMat.cpp:452-534.
//
// The reference writes the candidates to a text file, runs
//     python3 src/gpu_graph_generator.py <cands> <edges.bin> <minED> <maxGB>
// through system(), exits on a non-zero status, and loads the edge file with
// AdjList::Init + AdjList::FromBinaryFile (src/SparseMat.cpp:338-390).  Here
// the candidates are packed in memory, the graph is built by the library on
// the GPU, and AdjList is filled from the library's canonical adjacency:
// row x = lower neighbours ascending, then upper neighbours ascending, which
// is exactly the order FromBinaryFile builds from the (u<v, rows ascending,
// columns ascending) pair file.  RowsBySum, Codebook and the checkpoint files
// of the caller are untouched.
//
// This file is meant to be compiled INSIDE src/SparseMat.cpp, in place of the
// reference's FillAdjListGPU definition (the callers at :749 and :812 use its
// default arguments, so the definition keeps them); it relies on that file's
// includes (<vector>, <string>, <iostream>, <chrono>, <iomanip>) and on
// `using namespace std`.  Link with -lindexgen_cuda.
//
// Threads: the cluster worker pool (src/SparseMat.cpp:985-1010) calls this
// from up to `threads` workers at once.  They share ONE library context; the
// context serialises their device work.
//
// Differences that a caller can see:
//   * no temp_vectors_<id>.txt / temp_edges_<id>.bin files are written (an
//     inputFilename given by the caller is not read: the strings are already
//     in memory);
//   * maxGPUMemoryGB is not a tile-size knob here (the library sizes its own
//     workspaces and has no edge cap);
//   * binary-alphabet candidates (isBinary) of length <= 16 are packed like
//     quaternary ones (Levenshtein distance over {0,1} does not depend on the
//     alphabet size); longer words are rejected with an error;
//   * on failure the process exits with status 1, as the reference does when
//     its script fails (src/SparseMat.cpp:500-513), after printing the
//     library's message.
#include <cstdlib>
#include <mutex>

#include "indexgen_cuda.h"

namespace {

ig_ctx *IgSharedContext()
{
    static ig_ctx *ctx = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        if (ig_ctx_create(&ctx, 0) != IG_OK || !ctx) {
            std::cerr << "Error: libindexgen_cuda could not create a GPU context." << std::endl;
            std::exit(1);
        }
    });
    return ctx;
}

[[noreturn]] void IgFail(const char *what, ig_status s)
{
    std::cerr << "Error: libindexgen_cuda " << what << " failed: " << ig_status_string(s) << " ("
              << ig_last_error(IgSharedContext()) << ")" << std::endl;
    std::exit(1);
}

}  // namespace

void FillAdjListGPU(AdjList &adjList, const vector<string> &candidates, const int minED, long long int &matrixOnesNum,
                    const string &inputFilename = "", double maxGPUMemoryGB = 10.0, bool silent = false,
                    bool isBinary = false)
{
    (void)inputFilename;
    (void)maxGPUMemoryGB;
    const auto t0 = chrono::steady_clock::now();
    const int64_t n = (int64_t)candidates.size();
    const int len = n > 0 ? (int)candidates[0].size() : 1;
    if (n > 0 && (len < 1 || len > IG_MAX_LEN)) {
        std::cerr << "Error: libindexgen_cuda handles words of length 1.." << IG_MAX_LEN << ", got " << len
                  << (isBinary ? " (binary alphabet)" : "") << "." << std::endl;
        std::exit(1);
    }
    std::string text;
    text.reserve((size_t)(n * len));
    for (const string &s : candidates) {
        if ((int)s.size() != len) {
            std::cerr << "Error: candidates of different lengths (" << s.size() << " vs " << len << ")." << std::endl;
            std::exit(1);
        }
        text += s;
    }
    std::vector<uint32_t> words((size_t)n);
    int64_t bad = -1;
    ig_status s = ig_pack(text.data(), n, len, len, words.data(), &bad);
    if (s != IG_OK) {
        std::cerr << "Error: candidate " << bad << " is not a string over 0..3." << std::endl;
        std::exit(1);
    }
    ig_ctx *ctx = IgSharedContext();
    ig_graph *g = nullptr;
    if ((s = ig_graph_build(ctx, words.data(), (int32_t)n, len, minED, 0, &g)) != IG_OK)
        IgFail("graph build", s);
    int64_t edges = 0;
    ig_graph_stats(g, nullptr, &edges);
    std::vector<int64_t> adj_ptr((size_t)n + 1);
    std::vector<int32_t> adj((size_t)(2 * edges));
    if ((s = ig_graph_adjacency(g, adj_ptr.data(), adj.data())) != IG_OK) {
        ig_graph_free(g);
        IgFail("adjacency download", s);
    }
    ig_graph_free(g);
    adjList.Init((int)n);
    for (int64_t x = 0; x < n; ++x)
        for (int64_t k = adj_ptr[(size_t)x]; k < adj_ptr[(size_t)x + 1]; ++k)
            adjList.Set((int)x, adj[(size_t)k]);
    matrixOnesNum = 2 * edges;
    if (!silent) {
        const chrono::duration<double> dt = chrono::steady_clock::now() - t0;
        std::cout << "[C++] libindexgen_cuda: " << edges << " edges for " << n << " candidates in " << fixed
                  << setprecision(2) << dt.count() << "s" << endl;
    }
}
