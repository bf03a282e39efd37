"""Non-homogeneous boundary data (pp_set_face_values): Dirichlet values and
Neumann outward derivatives on any face.  The test builds a problem whose
discrete solution is known exactly: a smooth u at the cell centres, its
ghost values across each face, face data from the ghost-cell relations
(Dirichlet g = (u_ghost + u_0) / 2, Neumann g = (u_ghost - u_0) / h) and a
right-hand side equal to the 7-point operator applied with those ghosts.  The
solve must return u to round-off -- a size-independent check of the data's
scaling ((dz/dx)^2 on x faces, (dz/dy)^2 on y faces), signs and indexing."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _u(x, y, z):
    return np.sin(1.3 * x + 0.4) * np.cos(0.7 * y - 0.2) * np.exp(0.5 * z) + 0.3 * x * y - 0.2 * z


def _problem(nx, ny, nz, bc, box):
    dx = (box[1] - box[0]) / nx
    dy = (box[3] - box[2]) / ny
    dz = (box[5] - box[4]) / nz
    # cell centres with one ghost layer on every side: index 0 and n+1 are ghosts
    xs = box[0] + (np.arange(-1, nx + 1) + 0.5) * dx
    ys = box[2] + (np.arange(-1, ny + 1) + 0.5) * dy
    zs = box[4] + (np.arange(-1, nz + 1) + 0.5) * dz
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    U = _u(X, Y, Z)  # (nz+2, ny+2, nx+2)
    u = U[1:-1, 1:-1, 1:-1]
    cx, cy = (dz / dx) ** 2, (dz / dy) ** 2
    lap = (cx * (U[1:-1, 1:-1, :-2] - 2 * u + U[1:-1, 1:-1, 2:]) +
           cy * (U[1:-1, :-2, 1:-1] - 2 * u + U[1:-1, 2:, 1:-1]) +
           (U[:-2, 1:-1, 1:-1] - 2 * u + U[2:, 1:-1, 1:-1]))
    f = lap / dz ** 2
    # face data (x faces (nz, ny), y faces (nz, nx), z faces (ny, nx))
    ghost = [U[1:-1, 1:-1, 0], U[1:-1, 1:-1, -1], U[1:-1, 0, 1:-1], U[1:-1, -1, 1:-1], U[0, 1:-1, 1:-1],
             U[-1, 1:-1, 1:-1]]
    first = [u[:, :, 0], u[:, :, -1], u[:, 0, :], u[:, -1, :], u[0], u[-1]]
    h = [dx, dx, dy, dy, dz, dz]
    faces = {}
    for f_ in range(6):
        if bc[f_] == "D":
            faces[f_] = 0.5 * (ghost[f_] + first[f_])
        elif bc[f_] == "N":
            faces[f_] = (ghost[f_] - first[f_]) / h[f_]
    return u, f, faces


CASES = [(32, 24, 20, "DDDDDD"), (32, 24, 20, "NNDDDN"), (30, 20, 17, "DNNDND"), (16, 48, 12, "NDDNDD"),
         (48, 32, 16, "DDNNNN"), (24, 40, 10, "NNNNDN")]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("precision", [0, 1])
def test_face_values_give_the_exact_discrete_solution(case, precision):
    import pittpack_b200 as pp

    nx, ny, nz, bc = case
    box = (0.0, 1.0, -0.5, 1.0, 0.2, 1.0)
    u, f, faces = _problem(nx, ny, nz, bc, box)
    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(bc)
        M.setBox(box)
        M.setCoords(2)
        M.setOptions(compat_zero_mode=0, precision=precision, max_sweeps=2)
        for face, g in faces.items():
            M.setFaceValues(face, g)
        M.assignRhs(f)
        M.pittPack()
        P = M.getSolution()
    err = np.linalg.norm(P.real - u) / np.linalg.norm(u)
    assert err <= (1e-11 if precision == 0 else 1e-10), (bc, precision, err)
    assert np.abs(P.imag).max() == 0.0


def test_face_values_replace_and_clear():
    import pittpack_b200 as pp

    nx, ny, nz, bc = 16, 16, 8, "DDNNDD"
    box = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    u, f, faces = _problem(nx, ny, nz, bc, box)
    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(bc)
        M.setOptions(compat_zero_mode=0, dirichlet_lift=0)
        M.assignRhs(f)
        M.pittPack()
        P0 = M.getSolution().copy()          # homogeneous data
        for face, g in faces.items():
            M.setFaceValues(face, g)
        M.pittPack()
        assert np.linalg.norm(M.getSolution().real - u) / np.linalg.norm(u) <= 1e-11
        for face in faces:
            M.setFaceValues(face, None)      # cleared: back to homogeneous data
        M.pittPack()
        assert np.array_equal(M.getSolution(), P0)
        with pytest.raises(pp.PittPackError):
            M.setFaceValues(6, faces[0])
        with pytest.raises(pp.PittPackError):
            M.setFaceValues(0, np.zeros(3))
    with pp.make_Poisson(16, 16, 8) as M:
        M.assignBoundary("PPPPDD")
        with pytest.raises(pp.PittPackError) as e:
            M.setFaceValues(0, np.zeros((8, 16)))   # periodic face
        assert e.value.code == 19
