"""CPU model of the tcgen05 level-0 convolution's schedule (k_conv3_tc in
bcm-problems_b200/csrc/unet.cu).

The kernel's correctness rests on its index bookkeeping rather than on its
arithmetic:

- the output rows (y-lines) of a CTA form one contiguous range of the
  nz * ny rows, walked as one segment per z plane;
- input line y' feeds rows y'+1, y', y'-1 through one N = 144 MMA per z tap,
  into 48-column accumulator blocks kept in a ring of NB blocks at descending
  tensor-memory columns, split into two MMAs where the ring wraps;
- a row is released to the epilogue after its last input line, and a block is
  reused only after its previous row was released.

This test replays that schedule exactly as the MMA thread computes it, with
numpy products standing in for the MMAs.  It checks the invariants (MMA
widths, column ranges, release-before-reuse, which is what keeps the
kernel's waits deadlock-free) and that the assembled rows equal the oracle's
convolution.  The GPU test of the same kernel is
tests/test_gpu_unet.py::test_unet_forward_tensor_core_level_matches_oracle.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import unet_ref as U  # noqa: E402

NB = 5      # accumulator blocks in the ring (tc::NB)
NX = 128    # x-line = the MMA's M


def blk_col(q):
    return 48 * (NB - 1 - q % NB)


def cta_schedule(ny, nz, grid, cta):
    """Events of one CTA's MMA thread, in issue order: ("acquire", q),
    ("mma", z, y, col, j0, cnt), ("release", q, z, r)."""
    ev = []
    nrow = nz * ny
    r0, r1 = nrow * cta // grid, nrow * (cta + 1) // grid
    q0, rs = 0, r0
    while rs < r1:
        z, ya = divmod(rs, ny)
        re = min(r1, (z + 1) * ny)
        yb = re - z * ny
        l0, l1 = max(ya - 1, 0), min(yb, ny - 1)
        acq, done = ya, ya
        for y in range(l0, l1 + 1):
            rlo, rhi = max(y - 1, ya), min(y + 1, yb - 1)
            if acq <= rhi:
                ev.append(("acquire", q0 + rhi - ya))
                acq = rhi + 1
            jlo, nr = y + 1 - rhi, rhi - rlo + 1
            b0 = (q0 + rhi - ya) % NB
            n1 = min(nr, b0 + 1)
            n2 = nr - n1
            ev.append(("mma", z, y, 48 * (NB - 1 - b0), jlo, n1))
            if n2:
                ev.append(("mma", z, y, 0, jlo + n1, n2))
            last = yb - 1 if y == l1 else y - 1
            while done <= last:
                ev.append(("release", q0 + done - ya, z, done))
                done += 1
        q0 += yb - ya
        rs = re
    return ev


def run_model(x, w, grid):
    """Assemble the convolution of x [nz][ny][128][cin] with w [27][16][cin]
    through the kernel's schedule; returns out [nz][ny][128][16]."""
    nz, ny, nx, cin = x.shape
    assert nx == NX
    # B operand per z tap: rows (dy, dx, n), the N = 144 of one MMA
    wb = w.reshape(3, 3, 3, 16, cin).reshape(3, 144, cin)
    out = np.full((nz, ny, NX, 16), np.nan)
    for cta in range(grid):
        tmem = np.zeros((NX, NB * 48))
        released, acq_top = set(), -1
        for e in cta_schedule(ny, nz, grid, cta):
            if e[0] == "acquire":
                # one wait, on the newest row's block, covers every row up to it
                # (the epilogue frees blocks in row order); each ring slot's
                # previous row must already have been released by this thread,
                # else the kernel's wait for it never ends
                q = e[1]
                assert q > acq_top
                for qq in range(acq_top + 1, q + 1):
                    if qq >= NB:
                        assert qq - NB in released, (cta, qq)
                acq_top = q
            elif e[0] == "mma":
                _, z, y, col, j0, cnt = e
                assert cnt in (1, 2, 3) and 0 <= col and col + 48 * cnt <= NB * 48
                for dz in range(3):
                    zi = z + dz - 1
                    if not 0 <= zi < nz:
                        continue  # TMA reads zeros outside the grid
                    a = x[zi, y]                                  # [128][cin]
                    b = wb[dz, 48 * j0:48 * (j0 + cnt)]           # [48 cnt][cin]
                    tmem[:, col:col + 48 * cnt] += a @ b.T
            else:
                _, q, z, r = e
                c = blk_col(q)
                assert q <= acq_top
                t = tmem[:, c:c + 48].reshape(NX, 3, 16)          # T[x'][dx][n]
                o = t[:, 1].copy()
                o[1:] += t[:-1, 0]                                # T0[x - 1]
                o[:-1] += t[1:, 2]                                # T2[x + 1]
                assert np.isnan(out[z, r, 0, 0]), "row written twice"
                out[z, r] = o
                tmem[:, c:c + 48] = 0.0                            # zeroed for its next use
                released.add(q)
    return out


@pytest.mark.parametrize("ny,nz,cin,grid", [(1, 1, 16, 1), (5, 3, 16, 1), (5, 3, 32, 4), (16, 8, 16, 128),
                                            (7, 4, 32, 6), (12, 2, 16, 5), (3, 9, 32, 27)])
def test_tc_schedule_matches_oracle_conv(ny, nz, cin, grid):
    rng = np.random.default_rng(ny * 100 + nz * 10 + grid)
    x = rng.standard_normal((nz, ny, NX, cin))
    w = rng.standard_normal((27, 16, cin))
    got = run_model(x, w, min(grid, nz * ny))
    assert not np.isnan(got).any(), "some output row was never released"
    want = U.conv(x, w)
    assert np.allclose(got, want, rtol=1e-12, atol=1e-10)


def test_tc_schedule_mma_widths_and_wrap_splits():
    """Interior lines use one N = 144 MMA except where the ring wraps, where
    the three blocks split 1+2 or 2+1; every released row was acquired."""
    widths, splits = set(), 0
    for cta in range(7):
        ev = cta_schedule(40, 6, 7, cta)
        m = [e for e in ev if e[0] == "mma"]
        widths |= {e[5] for e in m}
        for a, b in zip(m, m[1:]):
            if a[1:3] == b[1:3]:
                splits += 1
                assert b[3] == 0 and a[5] + b[5] <= 3
    assert widths == {1, 2, 3}
    assert splits > 0


def test_tc_schedule_ring_too_small_is_caught(monkeypatch):
    """A ring of two blocks cannot hold the three rows a line feeds: the model
    catches the acquire of a block whose previous row is still unreleased
    (the kernel would wait on it forever); three blocks are the minimum."""
    rng = np.random.default_rng(0)
    x = rng.standard_normal((3, 7, NX, 16))
    w = rng.standard_normal((27, 16, 16))
    monkeypatch.setattr(sys.modules[__name__], "NB", 2)
    with pytest.raises(AssertionError):
        run_model(x, w, 2)
    monkeypatch.setattr(sys.modules[__name__], "NB", 3)
    assert np.allclose(run_model(x, w, 2), U.conv(x, w))
