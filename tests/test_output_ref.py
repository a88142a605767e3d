"""The checker of the dump files: the reference's own output() (src/output.cpp)
run through oracle/_ref/how_ref --output.  This pins what the GPU writer is
compared with: the appended arrays of the reference's .vts equal a numpy
restatement of its per-cell formulas (separately rounded operations in the
source's left-to-right order, no fused multiply-adds), its block headers and
offsets follow the layout [u64 bytes][payload] from the byte after "_", and
its .dat rows carry the same numbers in "%.15e" text."""
import struct
import subprocess

import numpy as np
import pytest

from howtest import REF_BIN, write_dump, write_input

needs_ref = pytest.mark.skipif(not REF_BIN.exists(), reason="reference build oracle/_ref/how_ref absent")


def _bc_index(idx, lo, hi, periodic):
    if periodic:
        return lo + (idx - lo) % (hi - lo + 1)
    return np.clip(idx, lo, hi)


def _expected(q, n, per, size, gam, gn=None, kofs=0):
    """Per-cell quantities of src/output.cpp:110-187, x fastest, for a block
    of n cells starting at global plane kofs of a gn grid (default: n, 0)."""
    nx, ny, nz = n
    gn = n if gn is None else gn
    i = np.arange(3, nx + 3)[None, None, :]
    j = np.arange(3, ny + 3)[None, :, None]
    k = np.arange(3, nz + 3)[:, None, None]
    d = [size[a] / gn[a] for a in range(3)]
    A = lambda v: q[v][3:nx + 3, 3:ny + 3, 3:nz + 3].transpose(2, 1, 0)   # (k, j, i)
    rho, Mx, My, Mz, Bx, By, Bz, E = (A(v) for v in range(8))
    vx, vy, vz = Mx / rho, My / rho, Mz / rho
    vv2 = (vx * vx + vy * vy) + vz * vz
    BB2 = (Bx * Bx + By * By) + Bz * Bz
    pg = (gam - 1.0) * ((E - (0.5 * rho) * vv2) - 0.5 * BB2)
    divB = np.zeros_like(rho)
    for ax, v, idx in ((0, 4, i), (1, 5, j), (2, 6, k)):
        if n[ax] <= 1:
            continue
        lo, hi = 3, n[ax] + 2
        m, p = _bc_index(idx - 1, lo, hi, per[ax]), _bc_index(idx + 1, lo, hi, per[ax])
        qa = q[v].transpose(2, 1, 0)   # (k, j, i)
        ka, ja, ia = np.broadcast_arrays(k, j, i)
        args_m, args_p = [ka, ja, ia], [ka, ja, ia]
        args_m[2 - ax] = np.broadcast_to(m, ka.shape)   # (k, j, i) position of this axis
        args_p[2 - ax] = np.broadcast_to(p, ka.shape)
        diff = qa[tuple(args_p)] - qa[tuple(args_m)]
        edge = np.broadcast_to((m == idx) | (p == idx), ka.shape)
        divB = divB + np.where(edge, diff / d[ax], diff / (2.0 * d[ax]))
    x = (np.arange(nx) + 0.5) * d[0]
    y = (np.arange(ny) + 0.5) * d[1]
    z = ((kofs + np.arange(nz)).astype(np.float64) + 0.5) * d[2]
    X, Y, Z = np.broadcast_arrays(x[None, None, :], y[None, :, None], z[:, None, None])
    vec = lambda a, b, c: np.stack([a, b, c], axis=-1).reshape(-1)
    return [rho.reshape(-1), pg.reshape(-1), E.reshape(-1), vv2.reshape(-1), BB2.reshape(-1),
            divB.reshape(-1), vec(vx, vy, vz), vec(Bx, By, Bz), vec(Mx, My, Mz), vec(X, Y, Z)]


def _run(tmp_path, n, bc, fmt, q, gam=5.0 / 3.0):
    kw = dict(nx=n[0], ny=n[1], nz=n[2], nt=1, tend=0.1, gam=gam, cour=0.4, problem="orszag_tang",
              x1bc=bc[0], x2bc=bc[1], x3bc=bc[2], output_format=fmt)
    inp = write_input(tmp_path / "in.in", **kw)
    write_dump(tmp_path / "state.bin", {"q": q})
    subprocess.run([str(REF_BIN), str(inp), "/dev/null", "--state", str(tmp_path / "state.bin"),
                    "--output", "5", "0.25"], cwd=tmp_path, check=True, capture_output=True, timeout=300)
    return (tmp_path / "output" / ("dump000005." + ("dat" if fmt == "dat" else "vts"))).read_bytes()


def _random_state(n, seed):
    rng = np.random.default_rng(seed)
    P = [a + 6 for a in n]
    q = rng.uniform(-1.0, 1.0, (8, *P))
    q[0] = rng.uniform(0.5, 2.0, P)
    q[7] = rng.uniform(5.0, 9.0, P)
    return q


@needs_ref
@pytest.mark.parametrize("n,bc", [((7, 5, 4), ("periodic", "open", "periodic")),
                                  ((9, 6, 1), ("open", "periodic", "periodic"))])
def test_reference_vts_is_the_restated_layout(tmp_path, n, bc):
    q = _random_state(n, 3)
    raw = _run(tmp_path, n, bc, "vts", q)
    head, _, rest = raw.partition(b'<AppendedData encoding="raw">\n_')
    offs = [int(t.split(b'"')[0]) for t in head.split(b'offset="')[1:]]
    per = [b == "periodic" for b in bc]
    exp = _expected(q, n, per, (1.0, 1.0, 1.0), 5.0 / 3.0)
    for off, e in zip(offs, exp):
        (nbytes,) = struct.unpack("<Q", rest[off:off + 8])
        assert nbytes == 8 * e.size
        got = np.frombuffer(rest[off + 8:off + 8 + nbytes], dtype="<f8")
        np.testing.assert_array_equal(got.view(np.uint64), e.astype("<f8").view(np.uint64))
    assert rest.endswith(b"\n  </AppendedData>\n</VTKFile>\n")


@needs_ref
def test_reference_dat_rows(tmp_path):
    n = (6, 4, 3)
    q = _random_state(n, 4)
    text = _run(tmp_path, n, ("periodic",) * 3, "dat", q).decode()
    lines = text.splitlines()
    assert lines[0] == "# step = 5" and lines[1] == "# time = 2.500000000000000e-01"
    rows = [ln for ln in lines if not ln.startswith("#")]
    assert len(rows) == 6 * 4 * 3
    exp = _expected(q, n, [True] * 3, (1.0, 1.0, 1.0), 5.0 / 3.0)
    rho, pg, divB = exp[0], exp[1], exp[5]
    for r, row in enumerate(rows):
        f = row.split(" ")
        assert len(f) == 22
        assert f[9] == "%.15e" % rho[r] and f[17] == "%.15e" % pg[r] and f[21] == "%.15e" % divB[r]


@needs_ref
@pytest.mark.parametrize("zbc", ["periodic", "open"])
def test_reference_piece_of_a_z_slab(tmp_path, zbc):
    """--piece R NZ KS runs the reference's writer with the local sizes and
    offsets an MPI rank of a z-split holds: the header names the rank, the
    global extent, the piece's extent and its global start; coordinates are
    global; the divB diagnostic wraps (or clamps) at the slab's own edges."""
    gn, r, k0, nzl = (6, 5, 9), 1, 4, 3
    q = _random_state(gn, 7)
    slab = q[:, :, :, k0:k0 + nzl + 6]
    bc = ("periodic", "open", zbc)
    kw = dict(nx=gn[0], ny=gn[1], nz=gn[2], nt=1, tend=0.1, gam=5.0 / 3.0, cour=0.4, problem="orszag_tang",
              x1bc=bc[0], x2bc=bc[1], x3bc=bc[2], output_format="vts")
    inp = write_input(tmp_path / "in.in", **kw)
    write_dump(tmp_path / "state.bin", {"q": slab})
    subprocess.run([str(REF_BIN), str(inp), "/dev/null", "--state", str(tmp_path / "state.bin"),
                    "--piece", str(r), str(nzl), str(k0), "--output", "5", "0.25"], cwd=tmp_path, check=True,
                   capture_output=True, timeout=300)
    raw = (tmp_path / "output" / "dump000005.vts").read_bytes()
    head, _, rest = raw.partition(b'<AppendedData encoding="raw">\n_')
    assert b'WholeExtent="0 5 0 4 0 8"' in head
    assert b'<Piece Extent="0 5 0 4 4 6">' in head
    assert b'Name="rank" NumberOfTuples="1" format="ascii">\n          1\n' in head
    assert b'format="ascii">\n          0 0 4\n' in head
    offs = [int(t.split(b'"')[0]) for t in head.split(b'offset="')[1:]]
    per = [b == "periodic" for b in bc]
    exp = _expected(slab, (gn[0], gn[1], nzl), per, (1.0, 1.0, 1.0), 5.0 / 3.0, gn=gn, kofs=k0)
    for off, e in zip(offs, exp):
        (nbytes,) = struct.unpack("<Q", rest[off:off + 8])
        got = np.frombuffer(rest[off + 8:off + 8 + nbytes], dtype="<f8")
        np.testing.assert_array_equal(got.view(np.uint64), e.astype("<f8").view(np.uint64))
