"""CPU enumeration of the shared-memory reads the kernels' conflict-free claims rest on.

Shared memory has 32 four-byte banks and serves 128 bytes per wavefront: a warp's 64-bit loads are
served per half-warp (16 lanes), its 128-bit loads per quarter-warp (8 lanes). A phase is free of bank
conflicts when its lanes touch distinct 8-byte (16-byte) slots of the 128-byte line, or the same
address.  The index arithmetic below restates, line for line, the kernels' own:
  * the FP64 TMA kernel's fragment offsets (nwchem-ccsd-trpdrv_b200/csrc/fused_tma.cu: perm8,
    kmajor_off, FragOffsets; lane group g = lane >> 2, t = lane & 3; warp sub-block rows rs*16 and
    columns cs*8), with the lane-label permutation read from that source file;
  * the energy walk over TMA-landed 16x16 tiles (nwchem-ccsd-trpdrv_b200/csrc/tengy_tile.cuh:
    swz128 and tengy_tile_pair_swz16: each half-warp walks one diagonal q = (r + d) mod 16) and its
    table of per-index vectors (tengy_tile_pair_swz16_sv)."""
import os
import re

import pytest

from conftest import ROOT

CSRC = os.path.join(ROOT, "nwchem-ccsd-trpdrv_b200", "csrc")


def _source(name):
    with open(os.path.join(CSRC, name)) as f:
        return f.read()


def _perm_constant():
    m = re.search(r"int perm8\(int g\)\s*\{\s*return\s*\((0x[0-9A-Fa-f]+)\s*>>\s*\(4 \* g\)\)\s*&\s*7;", _source("fused_tma.cu"))
    assert m, "perm8 not found in fused_tma.cu"
    return int(m.group(1), 16)


def _const(name, src="fused_tma.cu"):
    m = re.search(r"constexpr int " + name + r"\s*=\s*([^;]+);", _source(src))
    assert m, name
    return m.group(1).strip()


PERM_HEX = _perm_constant()
PANEL_BYTES = int(_const("PANEL_BYTES"))
KBOX = PANEL_BYTES // 2
assert _const("KBOX") == "PANEL_BYTES / 2"


def perm8(g):
    return (PERM_HEX >> (4 * g)) & 7


def kmajor_off(kk, x):
    h, xi = x >> 4, x & 15
    return h * KBOX + kk * 128 + (((xi >> 1) ^ (kk & 7)) << 4) + ((xi & 1) << 3)


def frag_offsets(rx0, cx0, g, t):
    r, c = rx0 + perm8(g), cx0 + perm8(g)
    return {
        "kA0": kmajor_off(2 * t, r), "kA1": kmajor_off(2 * t, r + 8),
        "kA2": kmajor_off(2 * t + 1, r), "kA3": kmajor_off(2 * t + 1, r + 8),
        "kB0": kmajor_off(2 * t, c), "kB1": kmajor_off(2 * t + 1, c),
        "xA0": r * 128 + ((t ^ (r & 7)) << 4), "xA1": (r + 8) * 128 + ((t ^ ((r + 8) & 7)) << 4),
        "xB": c * 128 + ((t ^ (c & 7)) << 4),
    }


def conflict_free(addrs, width):
    """One phase: distinct `width`-byte slots of the 128-byte line, or identical addresses."""
    slots = {}
    for a in addrs:
        assert a % width == 0
        s = (a % 128) // width
        if s in slots and slots[s] != a:
            return False
        slots[s] = a
    return True


def warp_origins():
    for warp in range(8):  # the 8 MMA warps
        rs = warp >> 2
        cs = (warp & 3) ^ (rs << 1)
        yield rs * 16, cs * 8


def test_permutation_is_a_permutation_of_the_eight_rows():
    assert sorted(perm8(g) for g in range(8)) == list(range(8))


@pytest.mark.parametrize("kind", ["kA0", "kA1", "kA2", "kA3", "kB0", "kB1"])
@pytest.mark.parametrize("second_kstep", [0, 1024])  # m16n8k16 reads the next 8 rows 1024 bytes further
def test_kmajor_fragment_loads_are_conflict_free(kind, second_kstep):
    for rx0, cx0 in warp_origins():
        offs = [frag_offsets(rx0, cx0, lane >> 2, lane & 3)[kind] + second_kstep for lane in range(32)]
        for half in (offs[:16], offs[16:]):  # 64-bit loads: two phases of 16 lanes
            assert conflict_free(half, 8), (kind, rx0, cx0, half)


@pytest.mark.parametrize("kind", ["xA0", "xA1", "xB"])
@pytest.mark.parametrize("kx", [0, 64])  # the second k-step of a 16-wide chunk: 64 bytes further
def test_xmajor_fragment_loads_are_conflict_free(kind, kx):
    for rx0, cx0 in warp_origins():
        offs = [frag_offsets(rx0, cx0, lane >> 2, lane & 3)[kind] ^ kx for lane in range(32)]
        for q in range(4):  # 128-bit loads: four phases of 8 lanes
            assert conflict_free(offs[8 * q:8 * q + 8], 16), (kind, rx0, cx0, kx, q)


def test_identity_labels_would_conflict():
    # the reason for the permutation: with row g for lane group g, a quarter-warp's two rows share
    # bit 2 and its 128-bit X-major reads land in the same four 16-byte slots
    def off(r, t):
        return r * 128 + ((t ^ (r & 7)) << 4)
    quarter = [off(g, t) for g in (0, 1) for t in range(4)]
    assert not conflict_free(quarter, 16)


def swz128(x, col):
    return (((x >> 1) ^ (col & 7)) << 1) | (x & 1)


@pytest.mark.parametrize("nthread", [128])  # the energy warps and the separate energy kernel
def test_energy_walk_reads_are_conflict_free(nthread):
    plane, box = 16 * 16, 8 * 16 * 16
    ndiag = 16 // (nthread // 16)
    for diag in (False, True):
        for f in range(8):
            for k in range(ndiag):
                for warp in range(nthread // 32):
                    bc, cb = [], []
                    for lane in range(32):
                        tid = 32 * warp + lane
                        r = tid & 15
                        d = (tid >> 4) + k * (nthread // 16)
                        q = (r + d) & 15
                        bc.append(8 * (f * plane + q * 16 + swz128(r, q)))                   # f_x(B + r, C + q)
                        cb.append(8 * ((0 if diag else box) + f * plane + r * 16 + swz128(q, r)))  # f_x(C + q, B + r)
                    for reads in (bc, cb):
                        for half in (reads[:16], reads[16:]):
                            assert conflict_free(half, 8), (diag, f, k, warp, half)


@pytest.mark.parametrize("nthread", [128])
def test_energy_vector_table_reads_are_conflict_free(nthread):
    # tengy_tile_pair_swz16_sv: rows of 16 doubles, side b at vsh[x * 16 + r], side c at
    # vsh[7 * 16 + x * 16 + q] for the seven per-index vectors x
    ndiag = 16 // (nthread // 16)
    for x in range(7):
        for k in range(ndiag):
            for warp in range(nthread // 32):
                vb, vc = [], []
                for lane in range(32):
                    tid = 32 * warp + lane
                    r = tid & 15
                    q = (r + (tid >> 4) + k * (nthread // 16)) & 15
                    vb.append(8 * (x * 16 + r))
                    vc.append(8 * (7 * 16 + x * 16 + q))
                for reads in (vb, vc):
                    for half in (reads[:16], reads[16:]):
                        assert conflict_free(half, 8), (x, k, warp, half)
