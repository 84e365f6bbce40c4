// The ball octree shared by the host builder (host.cpp) and the device
// builder (tree_dev.cu): the reference's fmm/octree.cpp tree over triangle
// bounding balls, nodes in depth-first preorder.
#pragma once

#include <cstdint>
#include <vector>

namespace tct {

struct OctNode {
    int64_t start, end;
    double c[3];
    double R;
    bool leaf;
    int depth;
    int64_t child[8];
};

struct Octree {
    std::vector<double> centers;   // tree order, 3 per ball
    std::vector<double> radii;     // tree order
    std::vector<int64_t> orig;     // tree position -> original index
    std::vector<OctNode> nodes;
};

}  // namespace tct

struct tct_tree {
    tct::Octree t;
    int max_height = 0;
    std::vector<int> height;
};
