// Test-infrastructure driver around the UNMODIFIED IndexGen reference sources.
//
// This file is part of the oracle (test infrastructure only).  It is linked
// against objects compiled from the reference's own src/*.cpp by
// oracle/Makefile and is used to (a) generate golden fixtures in this
// container and (b) time the reference CPU path as the baseline arm of
// bench.py.  Nothing in the product library links or calls it.
//
// Sub-commands (all outputs little-endian int32 unless stated):
//   gen    <config.json> <out.txt>           Candidates(params)  (src/Candidates.cpp:178)
//   adj    <cands.txt> <minED> <T> <out.bin> FillAdjList(T) neighbour lists m[] in the
//                                            reference's own order (src/SparseMat.cpp:567-615)
//                                            out = [N][deg_0 nbrs_0...][deg_1 ...]...
//   solve  <cands.txt> <minED> <T> <out.bin> FillAdjList(T) + RowsBySum + FindMinDel loop, the
//                                            body of SolveIndependentSet (src/SparseMat.cpp:784-851);
//                                            out = [count][selected vertex ids in order]
//   edges  <cands.txt> <minED> <T> <out.bin> sorted (i<j) pairs with !EditDistanceBandedAtLeast,
//                                            as Tests/consistency/dump_candidates_and_cpu_edges.cpp
//   gpuload <N> <pairs.bin> <out.bin>        AdjList::Init + FromBinaryFile + greedy (GPU-path assembly)
//   time   <cands.txt> <minED> <T>           FillAdjList(T) wall time; prints JSON
//   pred   <a> <b> <minED>                   prints EditDistanceBandedAtLeast(b, MakePattern(a), minED)
//   predfile <pairs.txt> <out.bin>           one line "a b minED" per query; out = uint8 per query
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

// Read access to AdjList::m (the neighbour order is the quantity under test).
#define private public
#include "SparseMat.hpp"
#undef private
#include "Candidates.hpp"
#include "EditDistance.hpp"
#include "IndexGen.hpp"
#include "Utils.hpp"

using namespace std;

// Free functions defined in src/SparseMat.cpp without a header declaration.
void FillAdjList(AdjList &adjList, const vector<string> &candidates, const int minED, const int threadNum,
                 const int saveInterval, const bool resume, long long int &matrixOnesNum);
vector<string> SolveIndependentSet(const vector<string> &candidates, const int minED, const int threadNum,
                                   const bool useGPU, double maxGPUMemoryGB, bool isBinary);

static vector<string> read_lines(const string &path)
{
    ifstream in(path);
    if (!in)
    {
        cerr << "cannot open " << path << "\n";
        exit(2);
    }
    vector<string> v;
    string line;
    while (getline(in, line))
    {
        while (!line.empty() && (line.back() == '\r' || line.back() == '\n' || line.back() == ' '))
            line.pop_back();
        if (!line.empty())
            v.push_back(line);
    }
    return v;
}

static void write_i32(const string &path, const vector<int32_t> &v)
{
    ofstream out(path, ios::binary);
    out.write(reinterpret_cast<const char *>(v.data()), v.size() * sizeof(int32_t));
}

int main(int argc, char **argv)
{
    if (argc < 2)
    {
        cerr << "usage: ref_driver gen|adj|solve|edges|time|pred ...\n";
        return 2;
    }
    string cmd = argv[1];
    if (cmd == "gen" && argc == 4)
    {
        Params params;
        LoadParamsFromJson(params, argv[2]);
        vector<string> c = Candidates(params);
        ofstream out(argv[3]);
        for (auto &s : c)
            out << s << '\n';
        cout << "{\"candidates\": " << c.size() << "}" << endl;
        return 0;
    }
    if (cmd == "pred" && argc == 5)
    {
        PatternHandle H = MakePattern(argv[2]);
        cout << (EditDistanceBandedAtLeast(argv[3], H, atoi(argv[4])) ? 1 : 0) << endl;
        return 0;
    }
    if (cmd == "predfile" && argc == 4)
    {
        ifstream in(argv[2]);
        string a, b;
        int k;
        vector<uint8_t> res;
        while (in >> a >> b >> k)
        {
            PatternHandle H = MakePattern(a);
            res.push_back(EditDistanceBandedAtLeast(b, H, k) ? 1 : 0);
        }
        ofstream out(argv[3], ios::binary);
        out.write(reinterpret_cast<const char *>(res.data()), res.size());
        return 0;
    }
    if (cmd == "gpuload" && argc == 5)
    {
        // The reference GPU path's assembly: AdjList::Init + FromBinaryFile of a
        // (u<v) int32 pair file (src/SparseMat.cpp:520-521), then RowsBySum and
        // the FindMinDel loop.  argv[2] = N (as text), argv[3] = pair file,
        // argv[4] = output.
        int N = atoi(argv[2]);
        AdjList adj;
        long long ones = 0;
        adj.Init(N);
        adj.FromBinaryFile(argv[3], ones, true);
        adj.RowsBySum();
        vector<bool> remaining(N, true);
        double d1 = 0, d2 = 0;
        vector<int32_t> sel;
        while (!adj.empty())
            sel.push_back(adj.FindMinDel(remaining, d1, d2));
        for (int i = 0; i < N; i++)
            if (remaining[i])
                sel.push_back(i);
        vector<int32_t> out;
        out.push_back((int32_t)sel.size());
        out.insert(out.end(), sel.begin(), sel.end());
        write_i32(argv[4], out);
        cout << "{\"N\": " << N << ", \"ones\": " << ones << ", \"codebook\": " << sel.size() << "}" << endl;
        return 0;
    }
    if (cmd == "tofile" && argc == 5)
    {
        // progress_adj_list.txt as the GPU path writes it: AdjList::Init +
        // FromBinaryFile of the pair file, then AdjList::ToFile (the first
        // SaveProgressCodebook of Codebook).  argv[2] = N, argv[3] = pair
        // file, argv[4] = output text.
        int N = atoi(argv[2]);
        AdjList adj;
        long long ones = 0;
        adj.Init(N);
        adj.FromBinaryFile(argv[3], ones, true);
        adj.ToFile(argv[4]);
        cout << "{\"N\": " << N << ", \"ones\": " << ones << "}" << endl;
        return 0;
    }
    if (cmd == "resume" && argc == 5)
    {
        // Codebook from a progress_adj_list.txt with every candidate still
        // remaining: AdjList::FromFile, the degree buckets (RowsBySum, which
        // the resume path needs before FindMinDel), the FindMinDel loop, then
        // the remaining candidates in id order.  argv[2] = candidate count N,
        // argv[3] = text file, argv[4] = output.
        int N = atoi(argv[2]);
        AdjList adj;
        adj.FromFile(argv[3]);
        adj.RowsBySum();
        vector<bool> remaining(N, true);
        double d1 = 0, d2 = 0;
        vector<int32_t> sel;
        while (!adj.empty())
            sel.push_back(adj.FindMinDel(remaining, d1, d2));
        for (int i = 0; i < N; i++)
            if (remaining[i])
                sel.push_back(i);
        vector<int32_t> out;
        out.push_back((int32_t)sel.size());
        out.insert(out.end(), sel.begin(), sel.end());
        write_i32(argv[4], out);
        cout << "{\"N\": " << N << ", \"codebook\": " << sel.size() << "}" << endl;
        return 0;
    }
    if (argc < 5)
    {
        cerr << "bad arguments\n";
        return 2;
    }
    vector<string> cands = read_lines(argv[2]);
    int minED = atoi(argv[3]);
    int T = atoi(argv[4]);
    if (cmd == "adj" && argc == 6)
    {
        AdjList adj;
        long long ones = 0;
        FillAdjList(adj, cands, minED, T, 0, false, ones);
        vector<int32_t> out;
        out.push_back((int32_t)adj.m.size());
        for (auto &row : adj.m)
        {
            out.push_back((int32_t)row.size());
            out.insert(out.end(), row.begin(), row.end());
        }
        write_i32(argv[5], out);
        cout << "{\"N\": " << cands.size() << ", \"ones\": " << ones << "}" << endl;
        return 0;
    }
    if (cmd == "solve" && argc == 6)
    {
        // Body of SolveIndependentSet with the selected vertex ids kept.
        AdjList adj;
        long long ones = 0;
        FillAdjList(adj, cands, minED, T, 0, false, ones);
        adj.RowsBySum();
        vector<bool> remaining(cands.size(), true);
        double d1 = 0, d2 = 0;
        vector<int32_t> sel;
        while (!adj.empty())
            sel.push_back(adj.FindMinDel(remaining, d1, d2));
        for (int i = 0; i < (int)remaining.size(); i++)
            if (remaining[i])
                sel.push_back(i);
        // Cross-check against the reference entry point itself (strings only).
        vector<string> cb = SolveIndependentSet(cands, minED, T, false, 1.0, false);
        bool same = cb.size() == sel.size();
        for (size_t i = 0; same && i < cb.size(); i++)
            same = (cb[i] == cands[sel[i]]);
        if (!same)
        {
            cerr << "SolveIndependentSet disagrees with the FindMinDel replay\n";
            return 3;
        }
        vector<int32_t> out;
        out.push_back((int32_t)sel.size());
        out.insert(out.end(), sel.begin(), sel.end());
        write_i32(argv[5], out);
        cout << "{\"N\": " << cands.size() << ", \"ones\": " << ones << ", \"codebook\": " << sel.size() << "}"
             << endl;
        return 0;
    }
    if (cmd == "edges" && argc == 6)
    {
        AdjList adj;
        long long ones = 0;
        FillAdjList(adj, cands, minED, T, 0, false, ones);
        vector<int32_t> out;
        for (int i = 0; i < (int)adj.m.size(); i++)
            for (int j : adj.m[i])
                if (i < j)
                    out.push_back(i), out.push_back(j);
        // rows are visited in order; sort the columns within each row
        vector<pair<int, int>> pr;
        pr.reserve(out.size() / 2);
        for (size_t k = 0; k < out.size(); k += 2)
            pr.push_back({out[k], out[k + 1]});
        sort(pr.begin(), pr.end());
        out.clear();
        for (auto &p : pr)
            out.push_back(p.first), out.push_back(p.second);
        write_i32(argv[5], out);
        cout << "{\"N\": " << cands.size() << ", \"ones\": " << ones << ", \"edges\": " << pr.size() << "}"
             << endl;
        return 0;
    }
    if (cmd == "time")
    {
        AdjList adj;
        long long ones = 0;
        auto t0 = chrono::steady_clock::now();
        FillAdjList(adj, cands, minED, T, 0, false, ones);
        adj.RowsBySum();
        auto t1 = chrono::steady_clock::now();
        double s = chrono::duration<double>(t1 - t0).count();
        long long n = (long long)cands.size();
        cout << "{\"N\": " << n << ", \"pairs\": " << n * (n - 1) / 2 << ", \"ones\": " << ones
             << ", \"seconds\": " << s << ", \"threads\": " << T << "}" << endl;
        return 0;
    }
    cerr << "unknown command or arguments\n";
    return 2;
}
