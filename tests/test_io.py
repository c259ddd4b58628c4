"""Matrix and vector files in the reference's formats (bsg_read_mtr_bin,
bsg_write_mtr_bin, bsg_read_mtr, bsg_read_vect, bsg_write_vect_bin,
bsg_read_vect_bin) against the reference's own readers and writers
(CSMatrixR::ReadMtrBin / WriteMtrBin / ReadMtr / ConvertToBinary,
Bslib/smatrixr.cpp:3852-4020; CSVector::ReadVect / WriteVectBin /
ReadVectBin, Bslib/svector.cpp:465-560).

The files are compared byte for byte and the arrays exactly; these are
host-side functions, so everything but the last test runs without a GPU.
The last one replays a system written by the reference on the GPU and
compares the solution with the reference's solve of the same file.
"""
import os

import numpy as np
import pytest

import problems as P


@pytest.fixture
def system():
    s = P.heat3d(6, 5, 4, sigma=1.0, seed=17)
    u = s.upper()
    norm = np.linspace(0.5, 2.0, s.n)
    return s, u, norm


def test_binary_system_matches_the_reference_writer(tmp_path, reflib, system):
    import bsg
    s, u, norm = system
    ours, theirs = str(tmp_path / "ours.bin"), str(tmp_path / "theirs.bin")
    bsg.write_system_bin(ours, u.ia, u.ja, u.a, [s.rhs[0], norm])
    reflib.write_system_bin(theirs, u.ia, u.ja, u.a, [s.rhs[0], norm])
    assert open(ours, "rb").read() == open(theirs, "rb").read()
    # the reference reads what we wrote, we read what the reference wrote
    ia, ja, a, (b, nv) = reflib.read_system_bin(ours, 2, s.n)
    assert np.array_equal(ia, u.ia) and np.array_equal(ja, u.ja) and np.array_equal(a, u.a)
    assert np.array_equal(b, s.rhs[0]) and np.array_equal(nv, norm)
    m, n, lst, ia, ja, a, (b, nv) = bsg.read_system_bin(theirs, 2)
    assert (m, n) == (s.n, s.n) and np.array_equal(lst, np.arange(s.n))
    assert np.array_equal(ia, u.ia) and np.array_equal(ja, u.ja) and np.array_equal(a, u.a)
    assert np.array_equal(b, s.rhs[0]) and np.array_equal(nv, norm)


def write_text_system(path, ia, ja, a, vecs):
    """The text layout CSMatrixR::ReadMtr and CSVector::ReadVect read: sizes,
    label lines, one number per line (values with 17 significant digits)."""
    with open(path, "w") as f:
        f.write(f"{len(ia) - 1}\n{ia[-1]}\nia\n")
        f.write("".join(f"{v}\n" for v in ia))
        f.write("ja\n")
        f.write("".join(f"{v}\n" for v in ja))
        f.write("matrix\n")
        f.write("".join(f"{v:.17g}\n" for v in a))
        for k, v in enumerate(vecs):
            f.write(f"vector {k}\n")
            f.write("".join(f"{x:.17g}\n" for x in v))


def test_text_conversion_matches_the_reference(tmp_path, reflib, system):
    """CSMatrixR::ConvertToBinary against our text readers + binary writers."""
    import bsg
    s, u, norm = system
    txt = str(tmp_path / "sys.txt")
    write_text_system(txt, u.ia, u.ja, u.a, [s.rhs[0], norm])
    theirs, ours = str(tmp_path / "theirs.bin"), str(tmp_path / "ours.bin")
    reflib.convert_to_binary(txt, theirs)
    n, ia, ja, a, (b, nv) = bsg.read_system_text(txt, 2)
    assert n == s.n and np.array_equal(ia, u.ia) and np.array_equal(ja, u.ja) and np.array_equal(a, u.a)
    assert np.array_equal(b, s.rhs[0]) and np.array_equal(nv, norm)
    bsg.write_system_bin(ours, ia, ja, a, [b, nv])
    assert open(ours, "rb").read() == open(theirs, "rb").read()


def test_sizes_query_leaves_the_offset(tmp_path, system):
    import ctypes as C
    import bsg
    s, u, norm = system
    path = str(tmp_path / "m.bin")
    bsg.write_system_bin(path, u.ia, u.ja, u.a, [s.rhs[0]])
    off = C.c_longlong(0)
    n, nz = C.c_int(), C.c_int()
    L = bsg.lib()
    assert L.bsg_read_mtr_bin(os.fsencode(path), C.byref(off), None, C.byref(n), None, C.byref(nz), None, None, None,
                              None) == bsg.OK
    assert off.value == 0 and n.value == s.n and nz.value == u.ia[-1]


def test_truncated_and_missing_files_are_errors(tmp_path, system):
    import bsg
    s, u, norm = system
    path = str(tmp_path / "m.bin")
    bsg.write_system_bin(path, u.ia, u.ja, u.a, [s.rhs[0]])
    data = open(path, "rb").read()
    cut = str(tmp_path / "cut.bin")
    with open(cut, "wb") as f:
        f.write(data[:len(data) // 2])
    with pytest.raises(bsg.BsgError) as e:
        bsg.read_system_bin(cut, 1)
    assert e.value.code == bsg.ERR_ARG and "cut.bin" in str(e.value)
    with pytest.raises(bsg.BsgError):
        bsg.read_system_bin(str(tmp_path / "absent.bin"), 0)
    with pytest.raises(bsg.BsgError):
        bsg.read_system_text(str(tmp_path / "absent.txt"), 0)


@pytest.mark.gpu
def test_replay_a_system_file_on_the_gpu(tmp_path, ctx, reflib):
    """A system the reference wrote (matrix, right-hand side, norm vector) is
    read back and solved on the GPU; the solution agrees with the
    reference's SolveSymm of the same arrays to 1e-8 relative."""
    import bsg
    s = P.heat3d(16, 14, 12, sigma=1.0, seed=19)
    u = s.upper()
    path = str(tmp_path / "dump.bin")
    reflib.write_system_bin(path, u.ia, u.ja, u.a, [s.rhs[0], np.ones(s.n)])
    m, n, lst, ia, ja, a, (b, _) = bsg.read_system_bin(path, 2)
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0, ittype=0, eps=1e-10, niter=2000)
    x = bsg.solve_symm(ctx, n, ia, ja, a, b, p)
    xr, info = reflib.solve_symm(u.ia, u.ja, u.a, s.rhs[0], fcttyp=2, tau1=1e-3, tau2=1e-3, memory=-1.0, ittype=0,
                                 eps=1e-10)
    assert np.linalg.norm(x - xr) <= 1e-8 * np.linalg.norm(xr)
