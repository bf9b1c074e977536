// metis_sort.cpp -- the reference's METIS vertex ordering for CEMAS banks, restated.
//
// TEST INFRASTRUCTURE ONLY.  Linked with METIS and GKlib compiled from the reference's own
// vendored sources (MeshProcess/External/{METIS,GKlib}) into oracle/_ref/libstg_metis.so by
// `make -C oracle ref`, and loaded by tests/test_metis_cpu.py to regenerate the shipped
// Assets/sorted_mesh/*.part files.  The product library never links or calls it.
//
// Follows MeshProcess/metis_partition/src:
//   * node_edge_model.cpp:5-28   METIS_PartGraphKway with default options (no vertex weights,
//                                edge weights = edge multiplicity), ncon = 1;
//   * mesh.cpp:486-549 (tets) and :551-600 (triangles)   the adjacency: for every element and
//                                every ordered pair of its vertices one count on the edge; a
//                                vertex's neighbours ascending (std::map order);
//   * metis_sort.cpp:71-110 (triangles), :231-270 (tets)   the slack loop: with s = 0, 1, ...
//                                nPart = (V + 16 - s - 1) / (16 - s) until no part exceeds 16;
//   * mesh.cpp:65-112            the order: (vertex, part) pairs sorted by part with std::sort
//                                (not stable), the sorted mesh's vertex i = pairs[i].vertex.
#include <algorithm>
#include <map>
#include <utility>
#include <vector>

#include <metis.h>

extern "C" int orc_metis_sort(int nv, int ne, int k, const int* elems, int block_size, int* part_out, int* order_out,
                              int* slack_out)
{
    if(nv < 1 || ne < 0 || (k != 3 && k != 4) || block_size < 2) return -1;
    // adjacency with multiplicities
    std::vector<std::map<idx_t, int>> adj((size_t)nv);
    for(int e = 0; e < ne; e++)
    {
        const int* v = elems + (size_t)e * k;
        for(int a = 0; a < k; a++)
            for(int b = 0; b < k; b++)
                if(a != b)
                {
                    if(v[a] < 0 || v[a] >= nv || v[b] < 0 || v[b] >= nv) return -1;
                    adj[(size_t)v[a]][v[b]] += 1;
                }
    }
    std::vector<idx_t> xadj((size_t)nv + 1, 0), adjncy, wgt;
    for(int i = 0; i < nv; i++) xadj[(size_t)i + 1] = xadj[(size_t)i] + (idx_t)adj[(size_t)i].size();
    adjncy.reserve((size_t)xadj.back());
    wgt.reserve((size_t)xadj.back());
    for(int i = 0; i < nv; i++)
        for(const auto& [j, w] : adj[(size_t)i])
        {
            adjncy.push_back(j);
            wgt.push_back(w);
        }

    std::vector<idx_t> part((size_t)nv, 0);
    int slack = 0;
    long nparts = 1;
    for(;; slack++)
    {
        if(slack >= block_size - 1) return -2;
        nparts = ((long)nv + block_size - slack - 1) / (block_size - slack);
        std::fill(part.begin(), part.end(), 0);
        if(nparts > 1)
        {
            idx_t n = nv, ncon = 1, np = (idx_t)nparts, objval = 0;
            if(METIS_PartGraphKway(&n, &ncon, xadj.data(), adjncy.data(), nullptr, nullptr, wgt.data(), &np, nullptr,
                                   nullptr, nullptr, &objval, part.data()) != METIS_OK)
                return -3;
        }
        std::vector<int> size((size_t)nparts, 0);
        for(int i = 0; i < nv; i++) size[(size_t)part[(size_t)i]]++;
        if(*std::max_element(size.begin(), size.end()) <= block_size) break;
    }

    std::vector<std::pair<idx_t, idx_t>> vp((size_t)nv);
    for(int i = 0; i < nv; i++) vp[(size_t)i] = {i, part[(size_t)i]};
    std::sort(vp.begin(), vp.end(), [](const auto& a, const auto& b) { return a.second < b.second; });
    for(int i = 0; i < nv; i++)
    {
        part_out[i] = part[(size_t)i];
        order_out[i] = vp[(size_t)i].first;
    }
    *slack_out = slack;
    return (int)nparts;
}
