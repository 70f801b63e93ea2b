// Stand-in for the reference's src/flute.hpp — TEST INFRASTRUCTURE ONLY.
//
// InstantGR's vendored FLUTE cannot run: its topology table POST9.dat is not
// shipped (it is listed in .MISSING_LARGE_BLOBS), and readLUT() exits when it
// is missing (src/flute.hpp:321-325).  oracle/Makefile builds the reference's
// main.cpp against this header instead (through a directory of links to the
// reference sources in which flute.hpp points here).  It offers the same
// contract (flute::Branch, flute::Tree, readLUT, flute(x, y, acc);
// src/flute.hpp:43-56, :1239) and answers with the Steiner provider of this
// project, so the reference and this project route the same trees.
#pragma once
#include <vector>

#include "steiner_core.hpp"

namespace flute {

typedef int DTYPE;

struct Branch {
    DTYPE x, y;
    int n;
};

struct Tree {
    int deg = 0;
    DTYPE length = 0;
    std::vector<Branch> branch;
    int branchCount() const { return deg * 2 - 2; }
};

inline void readLUT() {}
inline void deleteLUT() {}

inline Tree flute(const std::vector<int> &x, const std::vector<int> &y, int /*acc*/) {
    Tree t;
    const int d = (int)x.size();
    t.deg = d;
    if (d < 2) return t;
    igr_steiner::Tree st;
    igr_steiner::build(x, y, st);
    std::vector<igr_steiner::Branch> br;
    igr_steiner::to_branches(x, y, st, br);
    t.branch.resize(br.size());
    for (size_t i = 0; i < br.size(); i++) t.branch[i] = Branch{br[i].x, br[i].y, br[i].n};
    for (auto &e : st.edges)
        t.length += (st.x[e.first] > st.x[e.second] ? st.x[e.first] - st.x[e.second] : st.x[e.second] - st.x[e.first]) +
                    (st.y[e.first] > st.y[e.second] ? st.y[e.first] - st.y[e.second] : st.y[e.second] - st.y[e.first]);
    return t;
}

}  // namespace flute
