"""The shared-memory stages of the tensor-map-staged solver passes
(bluebottle_b200/csrc/bbb_krylov_async.cuh), checked on the CPU against the
layout constants the library was compiled with (bbb_stage_layout).

For every staged pass in both precisions and for periodic, walled and
ragged boxes (row counts that are not a multiple of the tile height, the
duplicated periodic face of the Helmholtz systems) the test replays what
one stage receives -- the tiled boxes of the halo arrays, the mask and the
own arrays, the x-wrap chunks and the y-wrap rows (as_issue) -- and what
every warp then reads from it (the offsets k_bicg_async computes for its
own rows, the rows south and north of them and the x-halo cells), and
requires that
  * every copied byte lands inside the stage and no byte is written twice
    (two asynchronous writes to one byte would race),
  * the bytes the stage's barrier is armed with equal the bytes copied,
  * every read finds the cell of the array its stencil needs (wrapped or
    clamped at the faces),
  * the resident blocks the pass targets fit in one SM's shared memory.
A read or copy outside the stage would fault the GPU; this is where such
a layout change is caught without one."""
import ctypes as C

import pytest

from bluebottle_b200 import abi

SMEM_PER_SM = 228 * 1024       # B200 shared memory per SM
SMEM_PER_BLOCK_RESERVED = 1024

NAMES = ("ESZ CH NA NO R TH WARPS THREADS BOXW BOXH ROWP OWNB EXT_OFF AREG "
         "MROWP MEXT_OFF MREG MASK_OFF OWN_OFF XW_OFF XWA STAGE NS SMEM "
         "TX_BASE TX_XSIDE TX_YSIDE MINB").split()

PASSES = [(0, 0), (0, 1), (0, 3), (1, 0), (1, 1), (1, 2), (1, 3)]

# (nx, ny, periodic x, periodic y, duplicated face x, duplicated face y)
BOXES = [(256, 32, 1, 1, 0, 0), (128, 33, 1, 1, 0, 1), (128, 32, 0, 0, 0, 0),
         (256, 17, 1, 0, 0, 0), (128, 9, 1, 1, 0, 0), (384, 40, 1, 1, 1, 1),
         (128, 1, 1, 1, 0, 0), (128, 2, 0, 1, 0, 0), (128, 31, 1, 1, 0, 0)]


def rup(v, a):
    return (v + a - 1) // a * a


def layout(fp64, pas):
    lib = abi.load()
    buf = (C.c_int * len(NAMES))()
    assert lib.bbb_stage_layout(fp64, pas, buf, len(NAMES)) == len(NAMES)
    return dict(zip(NAMES, buf))


def derived(L):
    """The stage layout from its free parameters, as the comment above
    as_layout states it: regions on 128-byte boundaries, TH + 2 box rows of
    [CH | 128 | CH] cells per halo array, two wrap rows, the mask alike in
    bytes, TH rows per own array, [2 sides][TH rows][16 B] x-wrap chunks."""
    esz, ch, na, no, th = L["ESZ"], L["CH"], L["NA"], L["NO"], L["TH"]
    d = {"BOXW": 128 + 2 * ch, "BOXH": th + 2, "MROWP": 160}
    d["ROWP"] = d["BOXW"] * esz
    d["OWNB"] = 128 * esz
    d["EXT_OFF"] = d["BOXH"] * d["ROWP"]
    d["AREG"] = rup(d["EXT_OFF"] + 2 * d["OWNB"], 128)
    d["MEXT_OFF"] = d["BOXH"] * 160
    d["MREG"] = rup(d["MEXT_OFF"] + 256, 128)
    d["MASK_OFF"] = na * d["AREG"]
    d["OWN_OFF"] = d["MASK_OFF"] + d["MREG"]
    d["XW_OFF"] = d["OWN_OFF"] + no * th * d["OWNB"]
    d["XWA"] = 2 * th * 16
    d["STAGE"] = rup(d["XW_OFF"] + (na + 1) * d["XWA"], 128)
    d["TX_BASE"] = na * d["BOXH"] * d["ROWP"] + d["BOXH"] * 160 + no * th * d["OWNB"]
    d["TX_XSIDE"] = (na + 1) * th * 16
    d["TX_YSIDE"] = na * d["OWNB"] + 128
    d["WARPS"] = th // L["R"]
    d["THREADS"] = 32 * d["WARPS"]
    return d


def replay(L, nx, ny, perx, pery, dupx, dupy):
    g = L.__getitem__
    esz, ch, na, no, R, TH = g("ESZ"), g("CH"), g("NA"), g("NO"), g("R"), g("TH")
    wW = (nx - 2 if dupx else nx - 1) if perx else 0
    wE = (1 if dupx else 0) if perx else nx - 1
    wS = (ny - 2 if dupy else ny - 1) if pery else 0
    wN = (1 if dupy else 0) if pery else ny - 1

    def cell(x, y):
        return (x, y) if 0 <= x < nx and 0 <= y < ny else None

    for i0 in range(0, nx, 128):
        for j0 in range(0, ny, TH):
            xl, xr, ys, yn = i0 == 0, i0 + 128 == nx, j0 == 0, j0 + TH >= ny
            st = {}

            def put(off, what, c, n):
                for e in range(n):
                    assert 0 <= off + e < g("STAGE"), (off + e, g("STAGE"))
                    assert off + e not in st, ("two copies write byte", off + e)
                    st[off + e] = (what + c) if c else None

            for a in range(na):                 # halo-array boxes
                for by in range(g("BOXH")):
                    for bx in range(g("BOXW")):
                        put(a * g("AREG") + by * g("ROWP") + bx * esz, ("h", a),
                            cell(i0 - ch + bx, j0 - 1 + by), esz)
            for by in range(g("BOXH")):         # mask box
                for bx in range(160):
                    put(g("MASK_OFF") + by * 160 + bx, ("m", 0),
                        cell(i0 - 16 + bx, j0 - 1 + by), 1)
            for b in range(no):                 # own-array boxes
                for by in range(TH):
                    for bx in range(128):
                        put(g("OWN_OFF") + (b * TH + by) * g("OWNB") + bx * esz,
                            ("o", b), cell(i0 + bx, j0 + by), esz)
            for side, on, gg in ((0, xl, wW), (1, xr, wE)):   # x-wrap chunks
                if not on:
                    continue
                d = g("XW_OFF") + side * TH * 16
                for a in range(na):
                    for by in range(TH):
                        for bx in range(ch):
                            put(d + a * g("XWA") + by * 16 + bx * esz, ("h", a),
                                cell(gg // ch * ch + bx, j0 + by), esz)
                for by in range(TH):
                    for bx in range(16):
                        put(d + na * g("XWA") + by * 16 + bx, ("m", 0),
                            cell(gg // 16 * 16 + bx, j0 + by), 1)
            for side, on, row in ((0, ys, wS), (1, yn, wN)):  # y-wrap rows
                if not on:
                    continue
                for a in range(na):
                    for x in range(128):
                        put(a * g("AREG") + g("EXT_OFF") + side * g("OWNB") + x * esz,
                            ("h", a), (i0 + x, row), esz)
                for x in range(128):
                    put(g("MASK_OFF") + g("MEXT_OFF") + side * 128 + x, ("m", 0),
                        (i0 + x, row), 1)
            armed = (g("TX_BASE") + (xl + xr) * g("TX_XSIDE")
                     + (ys + yn) * g("TX_YSIDE"))
            assert len(st) == armed, (len(st), armed)

            def rd(off, want, n):
                for e in range(n):
                    assert st.get(off + e, "never written") == want, \
                        (off + e, want, st.get(off + e, "never written"), i0, j0)

            for w in range(g("WARPS")):
                jw = j0 + R * w
                nv = min(R, ny - jw)
                if nv <= 0:
                    continue
                rb = R * w + 1
                nwrap = jw + nv == ny
                srow = wS if jw == 0 else jw - 1
                nrow = wN if nwrap else jw + nv
                for tx in range(32):
                    col = 4 * tx
                    h_own = rb * g("ROWP") + (ch + col) * esz
                    m_own = g("MASK_OFF") + rb * 160 + 16 + col
                    h_s = (g("EXT_OFF") + col * esz if jw == 0
                           else (rb - 1) * g("ROWP") + (ch + col) * esz)
                    m_s = (g("MASK_OFF") + g("MEXT_OFF") + col if jw == 0
                           else g("MASK_OFF") + (rb - 1) * 160 + 16 + col)
                    h_n = (g("EXT_OFF") + g("OWNB") + col * esz if nwrap
                           else (rb + R) * g("ROWP") + (ch + col) * esz)
                    m_n = (g("MASK_OFF") + g("MEXT_OFF") + 128 + col if nwrap
                           else g("MASK_OFF") + (rb + R) * 160 + 16 + col)
                    o_own = g("OWN_OFF") + R * w * g("OWNB") + col * esz
                    for v in range(4):
                        x = i0 + col + v
                        for a in range(na):
                            for r in range(nv):
                                rd(h_own + r * g("ROWP") + a * g("AREG") + v * esz,
                                   ("h", a, x, jw + r), esz)
                            rd(h_s + a * g("AREG") + v * esz, ("h", a, x, srow), esz)
                            rd(h_n + a * g("AREG") + v * esz, ("h", a, x, nrow), esz)
                        for r in range(nv):
                            rd(m_own + r * 160 + v, ("m", 0, x, jw + r), 1)
                            for b in range(no):
                                rd(o_own + (b * TH + r) * g("OWNB") + v * esz,
                                   ("o", b, x, jw + r), esz)
                        rd(m_s + v, ("m", 0, x, srow), 1)
                        rd(m_n + v, ("m", 0, x, nrow), 1)
                    if tx not in (0, 31):
                        continue
                    if tx == 0:
                        xc = wW if xl else i0 - 1
                        if xl:
                            h_x = g("XW_OFF") + R * w * 16 + (wW % ch) * esz
                            m_x = g("XW_OFF") + na * g("XWA") + R * w * 16 + wW % 16
                            xs, hr, mr = g("XWA"), 16, 16
                        else:
                            h_x = rb * g("ROWP") + (ch - 1) * esz
                            m_x = g("MASK_OFF") + rb * 160 + 15
                            xs, hr, mr = g("AREG"), g("ROWP"), 160
                    else:
                        xc = wE if xr else i0 + 128
                        if xr:
                            h_x = (g("XW_OFF") + TH * 16 + R * w * 16
                                   + (wE % ch) * esz)
                            m_x = (g("XW_OFF") + na * g("XWA") + TH * 16 + R * w * 16
                                   + wE % 16)
                            xs, hr, mr = g("XWA"), 16, 16
                        else:
                            h_x = rb * g("ROWP") + (ch + 128) * esz
                            m_x = g("MASK_OFF") + rb * 160 + 16 + 128
                            xs, hr, mr = g("AREG"), g("ROWP"), 160
                    for r in range(nv):
                        for a in range(na):
                            rd(h_x + r * hr + a * xs, ("h", a, xc, jw + r), esz)
                        rd(m_x + r * mr, ("m", 0, xc, jw + r), 1)


@pytest.mark.parametrize("fp64,pas", PASSES)
def test_compiled_layout_is_the_stated_one(fp64, pas):
    L = layout(fp64, pas)
    assert L["ESZ"] == (8 if fp64 else 4) and L["CH"] * L["ESZ"] == 16
    assert L["TH"] % L["R"] == 0
    for k, v in derived(L).items():
        assert L[k] == v, (k, L[k], v)
    assert (L["SMEM"] + SMEM_PER_BLOCK_RESERVED) * L["MINB"] <= SMEM_PER_SM
    # tensor-copy boxes: rows of a multiple of 16 bytes, at most 256 per side
    assert (L["BOXW"] * L["ESZ"]) % 16 == 0 and L["BOXH"] <= 256
    assert L["STAGE"] % 128 == 0 and L["AREG"] % 128 == 0


def test_unknown_pass_is_refused():
    lib = abi.load()
    buf = (C.c_int * len(NAMES))()
    assert lib.bbb_stage_layout(0, 2, buf, len(NAMES)) == -1
    assert lib.bbb_stage_layout(1, 4, buf, len(NAMES)) == -1
    assert lib.bbb_stage_layout(1, 0, buf, len(NAMES) - 1) == -1


@pytest.mark.parametrize("fp64,pas", PASSES)
def test_stage_copies_and_reads(fp64, pas):
    L = layout(fp64, pas)
    for box in BOXES:
        replay(L, *box)
