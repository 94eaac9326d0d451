"""The compile-time index tables of the Taylor kernels
(sumpy_b200/csrc/index_tables.cuh), checked on the host: the header is
compiled by nvcc into a small host program that prints every table for a
few orders, and each entry is compared with the multi-index formulas of
sumpy's coefficient orders (sumpy/expansion/__init__.py:643-752): the P2M
transposed-projection sweep (with its Helmholtz term), the packed L2P
decompression in the [(j, k)][i] layout, the full-layout shifts and
decompression of the Helmholtz L2L, the stored-coefficient maps, and the
16-byte alignment of the int4 arrays the kernels read (no GPU needed)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
NVCC = Path("/usr/local/cuda/bin/nvcc")
ORDERS = (0, 1, 2, 3, 6, 10, 14, 16)

PROGRAM = r"""
#include <cstdio>
#include <cstddef>
#include "index_tables.cuh"
using namespace sumpy;
template <int P> void dump()
{
    static constexpr P2mSweep<P> S{};
    static constexpr L2pDecomp<P> L{};
    static constexpr FullShift<P> T{};
    printf("order %d\n", P);
    printf("align %zu %zu %zu %zu %zu %zu\n", alignof(P2mSweep<P>), alignof(L2pDecomp<P>),
           alignof(FullShift<P>), offsetof(P2mSweep<P>, e), offsetof(L2pDecomp<P>, e),
           offsetof(FullShift<P>, e));
    printf("sweep_e"); for (int i = 0; i < 4 * P2mSweep<P>::NE; ++i) printf(" %d", S.e[i]); printf("\n");
    printf("sweep_start"); for (int i = 0; i < P + 2; ++i) printf(" %d", S.start[i]); printf("\n");
    printf("sweep_stored"); for (int i = 0; i < (P + 1) * (P + 1); ++i) printf(" %d", S.stored[i]); printf("\n");
    printf("l2p_e"); for (int i = 0; i < 4 * L2pDecomp<P>::NE; ++i) printf(" %d", L.e[i]); printf("\n");
    printf("l2p_start"); for (int i = 0; i < P + 2; ++i) printf(" %d", L.start[i]); printf("\n");
    printf("l2p_stored"); for (int i = 0; i < (P + 1) * (P + 1); ++i) printf(" %d", L.stored[i]); printf("\n");
    printf("shift_start"); for (int i = 0; i <= FullShift<P>::NFULL; ++i) printf(" %d", T.start[i]); printf("\n");
    for (int d = 0; d < 3; ++d) {
        printf("shift_idx%d", d);
        for (int i = 0; i < FullShift<P>::NT; ++i) printf(" %d", T.idx[d][i]);
        printf("\n");
    }
    printf("shift_e"); for (int i = 0; i < 4 * FullShift<P>::NE; ++i) printf(" %d", T.e[i]); printf("\n");
    printf("shift_dstart"); for (int i = 0; i < P + 2; ++i) printf(" %d", T.dstart[i]); printf("\n");
    printf("shift_sdeg"); for (int i = 0; i < (P + 1) * (P + 1); ++i) printf(" %d", T.sdeg[i]); printf("\n");
}
int main() { %DUMPS% return 0; }
"""


def full_index(i, j, k):
    d = i + j + k
    return d * (d + 1) * (d + 2) // 6 + i * (d + 1) - i * (i - 1) // 2 + j


def jki_offset(p, j, k):
    a = p + 1
    return (a * (a + 1) * (a + 2) // 6 - (a - j) * (a - j + 1) * (a - j + 2) // 6 + k * (a - j)
            - k * (k - 1) // 2)


def stored_set(p):
    out = []
    for d in range(p + 1):
        out += [(0, j, d - j) for j in range(d + 1)] + [(1, j, d - 1 - j) for j in range(d)]
    return out


@pytest.fixture(scope="module")
def tables(tmp_path_factory):
    if not NVCC.exists() or shutil.which("g++") is None:
        pytest.skip("nvcc / g++ not available")
    d = tmp_path_factory.mktemp("index_tables")
    src = d / "dump.cu"
    src.write_text(PROGRAM.replace("%DUMPS%", " ".join(f"dump<{p}>();" for p in ORDERS)))
    exe = d / "dump"
    subprocess.run([str(NVCC), "-std=c++17", "-I", str(ROOT / "include"),
                    "-I", str(ROOT / "sumpy_b200" / "csrc"), "-o", str(exe), str(src)],
                   check=True, capture_output=True, timeout=600)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    res, cur = {}, None
    for line in out.splitlines():
        key, *vals = line.split()
        if key == "order":
            cur = res.setdefault(int(vals[0]), {})
        else:
            cur[key] = [int(v) for v in vals]
    return res


@pytest.mark.parametrize("p", ORDERS)
def test_alignment(tables, p):
    a = tables[p]["align"]
    assert a[:3] == [16, 16, 16] and a[3:] == [0, 0, 0]


@pytest.mark.parametrize("p", ORDERS)
def test_p2m_sweep_and_stored_map(tables, p):
    t = tables[p]
    n, e = 0, t["sweep_e"]
    for pl, i in enumerate(range(p, 1, -1)):
        assert t["sweep_start"][pl] == n
        m = p - i + 2
        for J in range(m + 1):
            for K in range(m - J + 1):
                want = [full_index(i - 2, J, K),
                        full_index(i, J - 2, K) if J >= 2 else -1,
                        full_index(i, J, K - 2) if K >= 2 else -1,
                        full_index(i, J, K) if J + K <= p - i else -1]
                assert e[4 * n:4 * n + 4] == want
                n += 1
    assert all(s == n for s in t["sweep_start"][max(p - 1, 0):])
    assert t["sweep_stored"] == [full_index(*mi) for mi in stored_set(p)]


@pytest.mark.parametrize("p", ORDERS)
def test_l2p_decompression_and_stored_map(tables, p):
    t = tables[p]
    n, e = 0, t["l2p_e"]
    for pl, i in enumerate(range(2, p + 1)):
        assert t["l2p_start"][pl] == n
        m = p - i
        for J in range(m + 1):
            for K in range(m - J + 1):
                assert e[4 * n:4 * n + 3] == [jki_offset(p, J, K) + i,
                                              jki_offset(p, J + 2, K) + i - 2,
                                              jki_offset(p, J, K + 2) + i - 2]
                n += 1
    assert t["l2p_stored"] == [jki_offset(p, j, k) + i for i, j, k in stored_set(p)]


@pytest.mark.parametrize("p", ORDERS)
def test_full_layout_shifts_and_decompression(tables, p):
    t = tables[p]
    full = [(i, j, d - i - j) for d in range(p + 1) for i in range(d + 1)
            for j in range(d - i + 1)]
    assert [full_index(*m) for m in full] == list(range(len(full)))
    pos = 0
    for f, m in enumerate(full):
        assert t["shift_start"][f] == pos
        for q in range(p - sum(m) + 1):
            for d in range(3):
                mm = list(m)
                mm[d] += q
                assert t[f"shift_idx{d}"][pos] == full_index(*mm)
            pos += 1
    assert t["shift_start"][len(full)] == pos
    n, e = 0, t["shift_e"]
    for pl, i in enumerate(range(2, p + 1)):
        assert t["shift_dstart"][pl] == n
        m = p - i
        for J in range(m + 1):
            for K in range(m - J + 1):
                assert e[4 * n:4 * n + 4] == [full_index(i, J, K), full_index(i - 2, J + 2, K),
                                              full_index(i - 2, J, K + 2),
                                              full_index(i - 2, J, K)]
                n += 1
    assert t["shift_sdeg"] == [sum(mi) for mi in stored_set(p)]
