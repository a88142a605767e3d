"""Dump files through how_output against the reference's own output()
(src/output.cpp, compiled into oracle/_ref/how_ref): for the same q(0) the
.dat table and the binary .vts StructuredGrid must be the same bytes.  The
state is a seeded perturbation of a problem state with signed zeros planted
in the momenta, on periodic, open and mixed boundaries in 1-D, 2-D and 3-D,
so the divB diagnostic's wrap and clamp branches and the text rendering of
-0 are all exercised."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from howtest import REF_BIN, active, write_dump, write_input

pytestmark = pytest.mark.gpu

CASES = [
    ("orszag_tang", (24, 20, 1), ("periodic", "periodic", "periodic"), 5.0 / 3.0),
    ("mpi_smooth3d", (12, 10, 8), ("periodic", "open", "periodic"), 5.0 / 3.0),
    ("brio_wu", (40, 1, 1), ("open", "open", "open"), 2.0),
    ("mhd_rotor", (16, 18, 1), ("open", "open", "periodic"), 1.4),
]


def _state(hm, p, seed):
    q = hm.problem_state(p)
    rng = np.random.default_rng(seed)
    a = active(q, p.nx, p.ny, p.nz)
    a *= 1.0 + 0.03 * rng.standard_normal(a.shape)
    m = a[3]
    m[rng.random(m.shape) < 0.2] = -0.0
    return q


@pytest.mark.parametrize("fmt", ["dat", "vts", "vtk"])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_dump_is_the_reference_file(tmp_path, case, fmt):
    import how_mhd as hm
    prob, n, bc, gam = case
    kw = dict(nx=n[0], ny=n[1], nz=n[2], nt=1, tend=0.1, gam=gam, cour=0.4, problem=prob,
              x1bc=bc[0], x2bc=bc[1], x3bc=bc[2], output_format=fmt)
    p = hm.make_parameters(**kw)
    step, time = 37, 0.0123456789
    with hm.Domain(p) as d:
        d.set_state(_state(hm, p, 11))
        path = Path(d.output(step, time, tmp_path / "ours"))
        q0 = d.get_state(0)
    inp = write_input(tmp_path / "in.in", **kw)
    write_dump(tmp_path / "state.bin", {"q": q0})
    subprocess.run([str(REF_BIN), str(inp), "/dev/null", "--state", str(tmp_path / "state.bin"),
                    "--output", str(step), repr(time)], cwd=tmp_path, check=True, capture_output=True,
                   timeout=600)
    ext = "dat" if fmt == "dat" else "vts"
    ref = (tmp_path / "output" / f"dump{step:06d}.{ext}").read_bytes()
    ours = path.read_bytes()
    assert path.name == f"dump{step:06d}.{ext}"
    assert len(ours) == len(ref)
    assert ours == ref


def test_dump_in_slabs_equals_one_pass(tmp_path):
    """A grid whose payload is staged in several slabs of z planes writes the
    same file as the reference, which holds it all at once."""
    import how_mhd as hm
    kw = dict(nx=64, ny=64, nz=64, nt=1, tend=0.1, gam=5.0 / 3.0, cour=0.4, problem="blast3d_b",
              x1bc="periodic", x2bc="periodic", x3bc="periodic", output_format="vts")
    p = hm.make_parameters(**kw)
    with hm.Domain(p) as d:
        d.init_problem()
        d.run(0.0, 3)
        path = Path(d.output(3, 0.5, tmp_path / "ours"))
        q0 = d.get_state(0)
    inp = write_input(tmp_path / "in.in", **kw)
    write_dump(tmp_path / "state.bin", {"q": q0})
    subprocess.run([str(REF_BIN), str(inp), "/dev/null", "--state", str(tmp_path / "state.bin"),
                    "--output", "3", "0.5"], cwd=tmp_path, check=True, capture_output=True, timeout=600)
    assert path.read_bytes() == (tmp_path / "output" / "dump000003.vts").read_bytes()


def test_unknown_format_is_an_error(tmp_path):
    import how_mhd as hm
    p = hm.make_parameters(nx=8, ny=8, nz=1, nt=1, tend=0.1, problem="orszag_tang", output_format="hdf5")
    with hm.Domain(p) as d:
        d.init_problem()
        with pytest.raises(hm.HowError):
            d.output(0, 0.0, tmp_path)


@pytest.mark.parametrize("fmt", ["vts", "dat"])
def test_async_dump_overlaps_the_steps(tmp_path, fmt):
    """how_output_async of a state, then three steps while it is written:
    the file equals the synchronous dump of that state, and the steps equal
    a run without dumps, bit for bit."""
    import how_mhd as hm
    kw = dict(nx=40, ny=36, nz=32, nt=1, tend=100.0, gam=5.0 / 3.0, cour=0.4, problem="blast3d_b",
              rhomin=1e-6, pgmin=1e-6, output_format=fmt)
    p = hm.make_parameters(**kw)
    with hm.Domain(p) as d:
        d.init_problem()
        t, _, _ = d.run(0.0, 2)
        sync = Path(d.output(2, t, tmp_path / "sync"))
        path = Path(d.output_async(2, t, tmp_path / "async"))
        d.run(t, 3)
        d.output_wait()
        q = d.get_state(0)
        # a second dump reuses the buffers
        again = Path(d.output_async(5, 1.0, tmp_path / "again"))
        d.output_wait()
    with hm.Domain(p) as d:
        d.init_problem()
        t, _, _ = d.run(0.0, 2)
        d.run(t, 3)
        q_ref = d.get_state(0)
        ref5 = Path(d.output(5, 1.0, tmp_path / "ref5"))
    assert path.read_bytes() == sync.read_bytes()
    np.testing.assert_array_equal(q, q_ref)
    assert again.read_bytes() == ref5.read_bytes()


def test_format_none_writes_nothing(tmp_path):
    import how_mhd as hm
    p = hm.make_parameters(nx=8, ny=8, nz=1, nt=1, tend=0.1, problem="orszag_tang", output_format="none")
    with hm.Domain(p) as d:
        d.init_problem()
        assert d.output(0, 0.0, tmp_path / "o") is None
        assert d.output_async(1, 0.0, tmp_path / "o") is None
        d.output_wait()
    assert not (tmp_path / "o").exists()


def test_driver_writes_the_reference_dumps(tmp_path):
    """how_mhd_b200 writes output/dump000000 (the initial state, which equals
    the reference's initial condition bit for bit) and one dump per output
    interval; the initial one is the file the reference's driver writes."""
    exe = REF_BIN.parents[2] / "how-mhd-kokkos_b200" / "how_mhd_b200"
    kw = dict(nx=32, ny=32, nz=1, nt=2, tend=0.02, gam=5.0 / 3.0, cour=0.4, problem="orszag_tang",
              x1bc="periodic", x2bc="periodic", x3bc="periodic", output_format="vts")
    inp = write_input(tmp_path / "in.in", **kw)
    run = tmp_path / "ours"
    run.mkdir()
    subprocess.run([str(exe), str(inp)], cwd=run, check=True, capture_output=True, timeout=300)
    for s in range(3):
        assert (run / "output" / f"dump{s:06d}.vts").exists()
    subprocess.run([str(REF_BIN), str(inp), "/dev/null", "--output", "0", "0.0"], cwd=tmp_path, check=True,
                   capture_output=True, timeout=300)
    assert (run / "output" / "dump000000.vts").read_bytes() == (tmp_path / "output" / "dump000000.vts").read_bytes()


GROUP_CASES = [
    # (problem, grid, boundaries, parts)
    ("mpi_smooth3d", (12, 10, 9), ("periodic", "open", "periodic"), 3),
    ("blast3d_b", (16, 12, 14), ("periodic", "periodic", "open"), 2),
]


@pytest.mark.parametrize("fmt", ["vts", "dat"])
@pytest.mark.parametrize("case", GROUP_CASES, ids=[c[0] for c in GROUP_CASES])
def test_group_pieces_are_the_reference_ranks_files(tmp_path, case, fmt):
    """A z-decomposed group writes one piece per part, and each piece is the
    file the reference's MPI rank of that slab writes (its own output() run on
    the slab with the rank's nz, kstart and cart_rank), byte for byte:
    header fields, global indices and coordinates, and the divB diagnostic
    wrapped or clamped at the slab's own edges.  For .vts a PStructuredGrid
    master lists the pieces with extents that tile the whole extent."""
    import xml.etree.ElementTree as ET
    import how_mhd as hm
    prob, n, bc, parts = case
    kw = dict(nx=n[0], ny=n[1], nz=n[2], nt=1, tend=0.1, gam=5.0 / 3.0, cour=0.4, problem=prob,
              x1bc=bc[0], x2bc=bc[1], x3bc=bc[2], output_format=fmt)
    p = hm.make_parameters(**kw)
    step, time = 12, 0.0421
    q = _state(hm, p, 5)
    with hm.Group(p, parts) as g:
        g.set_state(q)
        master, pieces = g.output(step, time, tmp_path / "ours")
        ranges = [g.part_range(k) for k in range(parts)]
    inp = write_input(tmp_path / "in.in", **kw)
    ext = "dat" if fmt == "dat" else "vts"
    for r, (k0, nzl) in enumerate(ranges):
        assert Path(pieces[r]).name == f"dump{step:06d}_rank{r:06d}.{ext}"
        work = tmp_path / f"ref{r}"
        work.mkdir()
        write_dump(work / "state.bin", {"q": q[:, :, :, k0:k0 + nzl + 6]})
        subprocess.run([str(REF_BIN), str(inp), "/dev/null", "--state", str(work / "state.bin"),
                        "--piece", str(r), str(nzl), str(k0), "--output", str(step), repr(time)],
                       cwd=work, check=True, capture_output=True, timeout=600)
        ref = (work / "output" / f"dump{step:06d}.{ext}").read_bytes()
        assert Path(pieces[r]).read_bytes() == ref, r
    if fmt == "dat":
        assert master is None
        return
    root = ET.parse(master).getroot()
    assert root.get("type") == "PStructuredGrid"
    grid = root.find("PStructuredGrid")
    assert grid.get("WholeExtent") == f"0 {n[0] - 1} 0 {n[1] - 1} 0 {n[2] - 1}"
    got = [(pc.get("Extent"), pc.get("Source")) for pc in grid.findall("Piece")]
    want = [(f"0 {n[0] - 1} 0 {n[1] - 1} {k0} {k0 + nzl - 1}", f"dump{step:06d}_rank{r:06d}.vts")
            for r, (k0, nzl) in enumerate(ranges)]
    assert got == want
    # the master declares the arrays each piece holds, in the pieces' order
    piece = ET.fromstring(Path(pieces[0]).read_bytes().split(b"<AppendedData")[0] + b"</VTKFile>")
    names = [a.get("Name") for a in piece.iter("DataArray") if a.get("format") == "appended" and a.get("Name")]
    assert [a.get("Name") for a in grid.find("PPointData")] == names
