"""Algorithmic bytes of the ray query, per unit of counted work.

The trace kernel's counting variant (LRT_TRACE_COUNT_WORK) and the oracle
count the same units (TLAS node visits, BLAS node-pair visits, triangle tests,
voxel visits, ...).  Multiplying by the bytes one unit must read from memory
in the device layout gives the bytes a launch moves if nothing were cached;
divided by the kernel time that is the roofline numerator.  Cache reuse is
not subtracted, so coherent primary rays can exceed the HBM peak.
"""
import numpy as np

from ._abi import COUNTER_NAMES

# bytes per counted unit (device layout of csrc/device_layout.h)
BYTES_PER_UNIT = {
    "tlas_nodes": 32,      # BVHNode
    "instances": 100,      # geomId 4 + transformInv 64 + geometry-table entry 32
    "blas_pairs": 64,      # BVHNodePair, 4 x 16-byte loads
    "leaf_calls": 4,       # packed {start,count} of m_primIdCount
    "tri_tests": 48,       # {A, B-A, C-A} as 3 float4
    "bricks": 52,          # SdfSBSNode 16 + per-model SBS table 32 + brick occupancy word 4
    "voxels": 4,           # surface-voxel mask word of one march iteration
    "voxel_loads": 32,     # 8 fp32 corners of a dense brick (surface voxels only)
    "st_steps": 0,         # register-only
    "octree_leaves": 64,   # origNodes box 32 + 8 corner values 32
    "svs_leaves": 16,      # SdfSVSNode
    "hits": 0,
    "normals": 64,         # transformInvTransposed
}
RAY_BYTES = 32           # posAndNear + dirAndFar
HIT_BYTES = 32           # CRT_Hit
SBS_COLOUR_BYTES = 128   # 8 colour indices + 8 RGB triples per SBS hit (indexed layouts)


def algorithmic_bytes(counters, n_rays, sbs_colour_hits=0):
    c = np.asarray(counters, dtype=np.float64)
    per = np.array([BYTES_PER_UNIT[k] for k in COUNTER_NAMES], dtype=np.float64)
    return float((c * per).sum() + n_rays * (RAY_BYTES + HIT_BYTES) + sbs_colour_hits * SBS_COLOUR_BYTES)
