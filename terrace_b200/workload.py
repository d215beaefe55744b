"""Seeds of the synthetic workloads (shared by the benchmark and the
profiling cases so both run the same batches).

Update batch j of seed stream s is rMat(n, hash32(s) ^ j, ...), with the
reference's hash32 (include/rmat_util.h:44-52, Thomas Wang's 32-bit integer
hash; graph_bm draws one rMat generator per batch, src/graph_bm.cc:342)."""


def hash32(a: int) -> int:
    a &= 0xFFFFFFFF
    a = ((a + 0x7ED55D16) + (a << 12)) & 0xFFFFFFFF
    a = ((a ^ 0xC761C23C) ^ (a >> 19)) & 0xFFFFFFFF
    a = ((a + 0x165667B1) + (a << 5)) & 0xFFFFFFFF
    a = ((a + 0xD3A2646C) ^ (a << 9)) & 0xFFFFFFFF
    a = ((a + 0xFD7046C5) + (a << 3)) & 0xFFFFFFFF
    a = ((a ^ 0xB55A4F09) ^ (a >> 16)) & 0xFFFFFFFF
    return a


def batch_seed(stream: int, j: int) -> int:
    return hash32(stream) ^ j
