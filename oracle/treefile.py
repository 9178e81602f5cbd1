"""CPU oracle of the reference's dataset dump (test infrastructure only: the
tests compare the library's tree file with it; no product path calls it).

Restates GLVisitorGPUTrace::buildPerLeafData (HulkEngine/src/
GLVisitorGPUTrace.cpp:163-228) and GLVisitorGPUTrace::saveDataSetToFile
(HulkEngine/src/GLVisitorGPUTrace.cpp:638-674) with the record layouts of
GLVisitorGPUTrace.hpp:44-63 (LeafExtData, KdFileHeader), KDTreeNode
(HulkEngine/public/SharedStructs.hpp:113-137) and TriangleIndices
(SharedStructs.hpp:37-41): header, nodes, per-leaf records, then at a
512-byte boundary the per-leaf triangle indices and vertices, each leaf's
blocks padded to 32 entries. Padding entries, which the reference leaves
uninitialised, are zero here, as is the unused fourth index.
"""
from __future__ import annotations

import struct

import numpy as np

LEAF = 4
PER_LEAF_MULT = 32


def per_leaf_data(nodes4, leaf_polys, verts4, tris4):
    """(LeafExtData rows, per-leaf indices [N, 4], per-leaf vertices [M, 4])."""
    nodes4 = np.asarray(nodes4, np.uint32).reshape(-1, 4)
    ext, idx, lv = [], [], []
    n_idx = n_v = 0
    for n in nodes4:
        if int(n[0]) != LEAF:
            continue
        vmap = {}
        io, vo = n_idx, n_v
        for k in range(int(n[2])):
            t = int(leaf_polys[int(n[1]) + k])
            loc = []
            for v in range(3):
                g = int(tris4[t][v])
                if g not in vmap:
                    vmap[g] = len(vmap)
                    lv.append(np.asarray(verts4[g], np.float32))
                    n_v += 1
                loc.append(vmap[g])
            idx.append(loc + [0])
            n_idx += 1
        ni, nv = n_idx - io, n_v - vo
        ri = (ni + PER_LEAF_MULT - 1) & ~(PER_LEAF_MULT - 1)
        rv = (nv + PER_LEAF_MULT - 1) & ~(PER_LEAF_MULT - 1)
        idx.extend([[0, 0, 0, 0]] * (ri - ni))
        lv.extend([np.zeros(4, np.float32)] * (rv - nv))
        n_idx += ri - ni
        n_v += rv - nv
        ext.append((io, vo, rv, ri))
    idx = np.asarray(idx, np.uint32).reshape(-1, 4)
    lv = np.asarray(lv, np.float32).reshape(-1, 4)
    return np.asarray(ext, np.uint32).reshape(-1, 4), idx, lv


def dataset_bytes(nodes4, leaf_polys, verts4, tris4):
    """The file saveDataSetToFile writes for this tree and scene."""
    nodes4 = np.ascontiguousarray(nodes4, np.uint32).reshape(-1, 4)
    ext, idx, lv = per_leaf_data(nodes4, leaf_polys, verts4, tris4)
    hsize = 9 * 8
    tree_off, tree_size = hsize, nodes4.nbytes
    ext_off, ext_size = tree_off + tree_size, ext.nbytes
    idx_off = (ext_off + ext_size + 511) & ~511
    idx_size = idx.nbytes
    v_off, v_size = idx_off + idx_size, lv.nbytes
    head = struct.pack("<9Q", hsize, tree_size, tree_off, ext_size, ext_off, idx_size, idx_off, v_size, v_off)
    body = nodes4.tobytes() + ext.tobytes()
    body += b"\0" * (idx_off - ext_off - ext_size)
    return head + body + idx.tobytes() + lv.tobytes()
