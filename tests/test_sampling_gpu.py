"""Device-side sampling for the reference's applications: the windowed maximum of the free
surface with its node (apps/shoal_focus_mpi.cu:195-205 scan the downloaded state on the
host) and gauges at the nearest nodes (apps/tsunami_margin_mpi.cu:184-198), against the
same scans in numpy on the downloaded state."""
from __future__ import annotations

import numpy as np
import pytest

import sgnb
from cases import bump_case

pytestmark = pytest.mark.gpu


def first_argmax(a):
    return int(np.flatnonzero(a == a.max())[0])


@pytest.mark.parametrize("bc", [0, 1])
def test_eta_max_windows_and_gauges(bc):
    kw, U = bump_case(bc, Nx=13, Ny=7)
    with sgnb.SGN2DB200(precision=sgnb.FP64_FAST, **kw) as d:
        H = sgnb.setup_bathymetry(P=4, Nx=13, Ny=7, Lx=kw["Lx"], Ly=kw["Ly"],
                                  bathy_kind=kw["bathy_kind"], bathy_par=kw["bathy_par"],
                                  bc_x=bc, bc_y=bc)["Hnod"]
        x, y = d.node_coords()
        for state in ("initial", "evolved"):
            if state == "initial":
                d.upload(U)
            else:
                d.integrate_adaptive(0.0, 0.05, 0.5 * d.cfl_time_step(0.5))
            eta = d.download()[: d.Nd] - H
            v, n = d.eta_max()
            assert v == eta.max() and n == first_argmax(eta)
            for win in ((kw["Lx"] / 2, np.inf, -np.inf, np.inf),
                        (1.0, 4.0, 2.0, 5.5),
                        (x[17], x[17], y[17], y[17])):  # a single node, bounds inclusive
                m = (x >= win[0]) & (x <= win[1]) & (y >= win[2]) & (y <= win[3])
                v, n = d.eta_max(win)
                em = np.where(m, eta, -np.inf)
                assert v == em.max() and n == first_argmax(em), win
            v, n = d.eta_max((100.0, 101.0, 0.0, 1.0))  # outside the domain
            assert n == -1 and v == -np.inf
            rng = np.random.default_rng(3)
            gx, gy = rng.uniform(0, kw["Lx"], 6), rng.uniform(0, kw["Ly"], 6)
            nodes = [d.nearest_node(px, py) for px, py in zip(gx, gy)]
            ref = [int(np.argmin((x - px) ** 2 + (y - py) ** 2)) for px, py in zip(gx, gy)]
            assert nodes == ref
            assert np.array_equal(d.sample_eta(nodes), eta[nodes])
        with pytest.raises(sgnb.SgnbError):
            d.sample_eta([d.Nd])


def _scratch(name):
    import os

    d = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_tmp")
    os.makedirs(d, exist_ok=True)
    return os.path.join(d, name)


def vtk_text(Nx, Ny, hx, hy, means):
    """The reference writer's text (src/io/vtk2d.h:46-82) from element means [5, Ny, Nx]."""
    out = ["# vtk DataFile Version 3.0\nSGN2D element means\nASCII\n",
           f"DATASET STRUCTURED_POINTS\nDIMENSIONS {Nx} {Ny} 1\n",
           "ORIGIN %.6f %.6f 0\nSPACING %.6f %.6f 1\n" % (0.5 * hx, 0.5 * hy, hx, hy),
           f"POINT_DATA {Nx * Ny}\n"]
    for name, f in zip(("eta", "u", "v", "p", "H"), means):
        out.append(f"SCALARS {name} float 1\nLOOKUP_TABLE default\n")
        for row in f:
            out.append("".join("%.5e " % v for v in row) + "\n")
    return "".join(out)


@pytest.mark.parametrize("bc", [0, 1])
def test_element_means_and_vtk(bc):
    """Element means as the reference's writer forms them (s += qw[a] qw[b] f, 0.25 s)
    and the legacy-VTK frame, compared with the reference's own writer (periodic case,
    compiled reference) and with the same scan in numpy."""
    import oracle as O

    kw, U = bump_case(bc, Nx=9, Ny=7)
    o = O.Oracle(**kw)
    qw = o.tables()["qw"]
    H = o.bathymetry()["Hnod"]
    Nd, ne = o.Nd, 9 * 7
    fields = [U[:Nd] - H, U[Nd:2 * Nd] / U[:Nd], U[2 * Nd:3 * Nd] / U[:Nd],
              U[4 * Nd:] / U[:Nd], H]
    ref = []
    for f in fields:
        f = f.reshape(ne, 25)
        s = np.zeros(ne)
        for b in range(5):
            for a in range(5):
                s = s + qw[a] * qw[b] * f[:, a + 5 * b]
        ref.append((0.25 * s).reshape(7, 9))
    ref = np.array(ref)
    with sgnb.SGN2DB200(precision=sgnb.FP64_EXACT, **kw) as d:
        d.upload(U)
        m = d.element_means()
        assert np.array_equal(m, ref)
        path = _scratch(f"frame_{bc}.vtk")
        d.write_vtk(path)
        text = open(path).read()
    assert text == vtk_text(9, 7, kw["Lx"] / 9, kw["Ly"] / 7, ref)
    if bc == 0 and O.reference_available():
        rpath = _scratch("frame_ref.vtk")
        O.Oracle(reference=True, **kw).write_vtk(U, rpath)
        assert open(rpath).read() == text
