"""Host-side mirror of the reference's solver interface over the C ABI.

``solver_SMG`` and ``solver_SOR`` keep the argument list and meaning of
include/solverFuncs.hpp:26-37 and :169-180 (numpy (ni+2, nj+2) float64
arrays indexed [i][j], block tables i_bl/j_bl of shape (n_bl, 2) or longer,
n_bl, iteration cap, tolerance, message flag, in/out solution).  As in the
reference, only the grid cells of ``solution`` are written and
non-convergence is not an exception: the returned ``Status`` says what
happened (the reference returns nothing).  Argument, CUDA and allocation
failures raise ``CathodeError``.

``Grid`` exposes the device-resident path: device planes in the library
layout (torch tensors of shape (nj+2, ld) on the grid's device), solved
without host round trips.
"""
from __future__ import annotations

import ctypes
from typing import Dict, Tuple

import numpy as np

from . import capi


def _ptr(a) -> int:
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()  # torch tensor


def _as_ij(a: np.ndarray, ni: int, nj: int, name: str) -> np.ndarray:
    a = np.asarray(a)
    if a.shape != (ni + 2, nj + 2):
        raise ValueError(f"{name}: expected shape {(ni + 2, nj + 2)}, got {a.shape}")
    return np.ascontiguousarray(a, dtype=np.float64)


class Grid:
    """A cth_grid: block union, device mask and multigrid hierarchy."""

    def __init__(self, ni: int, nj: int, i_bl, j_bl, n_bl: int | None = None, device: int = 0):
        L = capi.load()
        ib = np.ascontiguousarray(np.asarray(i_bl, dtype=np.int32).reshape(-1, 2))
        jb = np.ascontiguousarray(np.asarray(j_bl, dtype=np.int32).reshape(-1, 2))
        if n_bl is None:
            n_bl = ib.shape[0]
        if n_bl > ib.shape[0] or n_bl > jb.shape[0] or n_bl < 1:
            raise ValueError("n_bl exceeds the block tables")
        ib = np.ascontiguousarray(ib[:n_bl])
        jb = np.ascontiguousarray(jb[:n_bl])
        h = ctypes.c_void_p()
        capi.check(L.cth_grid_create(ni, nj, ib.ctypes.data_as(capi._ip), jb.ctypes.data_as(capi._ip),
                                     n_bl, device, ctypes.byref(h)), allow_positive=False)
        self._h = h
        self._L = L
        self.ni, self.nj, self.n_bl, self.device = ni, nj, n_bl, device
        self.i_bl, self.j_bl = ib, jb
        self.ld = L.cth_grid_ld(h)
        self.levels = L.cth_grid_levels(h)

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._L.cth_grid_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def launch_count(self) -> int:
        return int(self._L.cth_launch_count(self._h))

    def profile(self, enable: bool = True):
        capi.check(self._L.cth_profile(self._h, int(enable)), allow_positive=False)

    def profile_read(self, cls: int):
        ms = ctypes.c_double()
        n = ctypes.c_longlong()
        by = ctypes.c_double()
        capi.check(self._L.cth_profile_read(self._h, cls, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(by)),
                   allow_positive=False)
        return ms.value, n.value, by.value

    def set_graphs(self, enable: bool):
        capi.check(self._L.cth_grid_set_graphs(self._h, int(enable)), allow_positive=False)

    def set_tail(self, enable: bool):
        """Fused coarse tail (levels of at most 16 rows in one cluster launch) on / off (default off)."""
        capi.check(self._L.cth_grid_set_tail(self._h, int(enable)), allow_positive=False)

    def time_cycle(self, precision: int, reps: int = 20, with_update: bool = True) -> float:
        """µs per multigrid cycle of ``reps`` cycles captured one after another in one
        graph without the solve's loop node (with or without the FP64 update)."""
        us = ctypes.c_double()
        capi.check(self._L.cth_grid_time_cycle(self._h, precision, reps, int(with_update), ctypes.byref(us)),
                   allow_positive=False)
        return us.value

    def set_reuse(self, tol: float, slot: int = -1):
        """Hierarchy reuse: with tol > 0 a solve given a slot keeps its multigrid
        hierarchy while the largest row-relative change of its operator stays at
        most tol (the time step's sweeps use their own slots; ``slot`` is the slot
        of the solves called on this grid directly, -1 none).  tol = 0: rebuild in
        every solve (default)."""
        capi.check(self._L.cth_grid_set_reuse(self._h, float(tol), int(slot)), allow_positive=False)

    def reuse_stats(self, precision: int, slot: int) -> dict:
        """Set-ups, reuses, last measured operator change, last cycle count and retries
        (rebuilds after a slow cycle on the kept hierarchy) of a slot."""
        out = (ctypes.c_double * 5)()
        capi.check(self._L.cth_grid_reuse_stats(self._h, precision, slot, out), allow_positive=False)
        return dict(setups=int(out[0]), reuses=int(out[1]), change=out[2], iterations=int(out[3]),
                    retries=int(out[4]))

    def time_relax(self, precision: int, level: int = 0, reps: int = 50):
        """(µs per launch, algorithmic bytes per launch) of one level's z-line
        relaxation, back-to-back in a graph as inside a cycle."""
        us, by = ctypes.c_double(), ctypes.c_double()
        capi.check(self._L.cth_grid_time_relax(self._h, precision, level, reps, ctypes.byref(us), ctypes.byref(by)),
                   allow_positive=False)
        return us.value, by.value

    def set_preconditioner(self, mode: int):
        """0: block Jacobi (the fields' V-cycles side by side, default); 1: block
        Gauss-Seidel across Ex, Er, Ephi."""
        capi.check(self._L.cth_mw3_set_preconditioner(self._h, int(mode)), allow_positive=False)

    def set_cycle(self, nu_pre: int, nu_post: int):
        capi.check(self._L.cth_grid_set_cycle(self._h, nu_pre, nu_post), allow_positive=False)

    # -- host-array solves (reference layout) ------------------------------
    def smg_solve(self, aP, aE, aW, aN, aS, b, solution, maxITR=30, error_cnv=1e-10,
                  precision=capi.CTH_PREC_FP64) -> capi.Status:
        ni, nj = self.ni, self.nj
        arrs = [_as_ij(a, ni, nj, n) for a, n in zip((aP, aE, aW, aN, aS, b), "aP aE aW aN aS b".split())]
        if not (isinstance(solution, np.ndarray) and solution.dtype == np.float64 and
                solution.flags.c_contiguous and solution.shape == (ni + 2, nj + 2)):
            raise ValueError("solution must be a C-contiguous float64 (ni+2, nj+2) array")
        st = capi.Status()
        rc = self._L.cth_smg_solve(self._h, *[a.ctypes.data for a in arrs], maxITR, error_cnv, precision,
                                   solution.ctypes.data, ctypes.byref(st))
        capi.check(rc)
        return st

    def sor_solve(self, aP, aE, aW, aN, aS, b, solution, alpha_SOR=1.9, maxITR=2000,
                  error_cnv=1e-8) -> capi.Status:
        ni, nj = self.ni, self.nj
        arrs = [_as_ij(a, ni, nj, n) for a, n in zip((aP, aE, aW, aN, aS, b), "aP aE aW aN aS b".split())]
        if not (isinstance(solution, np.ndarray) and solution.dtype == np.float64 and
                solution.flags.c_contiguous and solution.shape == (ni + 2, nj + 2)):
            raise ValueError("solution must be a C-contiguous float64 (ni+2, nj+2) array")
        st = capi.Status()
        rc = self._L.cth_sor_solve(self._h, *[a.ctypes.data for a in arrs], alpha_SOR, maxITR, error_cnv,
                                   solution.ctypes.data, ctypes.byref(st))
        capi.check(rc)
        return st

    def c5_solve(self, aP, aE, aW, aN, aS, b, solution, maxITR=500, error_cnv=1e-10) -> capi.Status:
        """Complex 5-point solve (host complex128 (ni+2, nj+2) arrays, [i][j])."""
        ni, nj = self.ni, self.nj
        arrs = []
        for a, n in zip((aP, aE, aW, aN, aS, b), "aP aE aW aN aS b".split()):
            a = np.asarray(a)
            if a.shape != (ni + 2, nj + 2):
                raise ValueError(f"{n}: expected shape {(ni + 2, nj + 2)}")
            arrs.append(np.ascontiguousarray(a, dtype=np.complex128))
        if not (isinstance(solution, np.ndarray) and solution.dtype == np.complex128 and
                solution.flags.c_contiguous and solution.shape == (ni + 2, nj + 2)):
            raise ValueError("solution must be a C-contiguous complex128 (ni+2, nj+2) array")
        st = capi.Status()
        rc = self._L.cth_c5_solve(self._h, *[a.ctypes.data for a in arrs], maxITR, error_cnv,
                                  solution.ctypes.data, ctypes.byref(st))
        capi.check(rc)
        return st

    def c5_solve_dev(self, aP, aE, aW, aN, aS, b, solution, maxITR=500, error_cnv=1e-10,
                     stream=None) -> capi.Status:
        """Complex 5-point solve on device planes (torch complex128, shape (nj+2, ld))."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        st = capi.Status()
        rc = self._L.cth_c5_solve_dev(self._h, *[_ptr(a) for a in (aP, aE, aW, aN, aS, b)], maxITR,
                                      error_cnv, _ptr(solution), s.cuda_stream, ctypes.byref(st))
        capi.check(rc)
        return st

    def impedance_test(self, epsr, params: dict, E1r, maxITR=400, error_cnv=1e-12, stream=None) -> dict:
        """The reference's impedance test (solve_Microwave_impedanceTest, emfieldModule.hpp:5528-6099)
        on this grid (single block: the Er faces [1, ni] x [2, nj]): assembly, solve, ghosts, port
        and rescale to Pmw on the device.  epsr: real device plane; E1r: torch complex128 (nj+2, ld),
        written in place.  params: dx, dr, rmin, omegam, J1r_exc, r1, r2, Z0, Pmw."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        prm = capi.ImpedanceParams(**{k: float(params[k]) for k, _ in capi.ImpedanceParams._fields_})
        res = capi.ImpedanceResult()
        rc = self._L.cth_mw_impedance_test(self._h, _ptr(epsr), ctypes.byref(prm), int(maxITR), float(error_cnv),
                                           _ptr(E1r), s.cuda_stream, ctypes.byref(res))
        capi.check(rc)
        return dict(V=complex(res.V[0], res.V[1]), I=complex(res.I[0], res.I[1]), P_fwd=res.P_fwd, P_ref=res.P_ref,
                    ratio=res.ratio, J1r_exc_factor=res.J1r_exc_factor, solve=res.solve.as_dict())

    def mw_divergence(self, E1x, E1r, E1p, J1x, J1r, J1p, dx, dr, rmin, omegam, stream=None):
        """output_phase's divE, divJ, div(E + J) columns (outputModule.hpp:43-105) on this
        grid's cells: torch complex128 (nj+2, ld) planes in; returns (divE, divJ, divEJ, Emag_rep)."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        out = [torch.zeros((self.nj + 2, self.ld), dtype=torch.complex128, device=f"cuda:{self.device}")
               for _ in range(3)]
        rep = ctypes.c_double()
        rc = self._L.cth_mw_divergence(self._h, *[_ptr(a) for a in (E1x, E1r, E1p, J1x, J1r, J1p)], float(dx),
                                       float(dr), float(rmin), float(omegam), *[_ptr(a) for a in out],
                                       ctypes.byref(rep), s.cuda_stream)
        capi.check(rc)
        return out[0], out[1], out[2], rep.value

    def mw_er_assemble_dev(self, ne, nu, epsr, params: dict, stream=None):
        """Er system of the microwave path on the device: returns complex planes
        (aP, aE, aW, aN, aS, b), each torch complex128 of shape (nj+2, ld)."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        out = [torch.zeros((self.nj + 2, self.ld), dtype=torch.complex128, device=f"cuda:{self.device}")
               for _ in range(6)]
        prm = capi.MWParams(**{k: float(params[k]) for k, _ in capi.MWParams._fields_})
        capi.check(self._L.cth_mw_er_assemble_dev(self._h, _ptr(ne), _ptr(nu), _ptr(epsr), ctypes.byref(prm),
                                                  *[_ptr(o) for o in out], s.cuda_stream), allow_positive=False)
        return out

    # -- device-resident path (library layout) -----------------------------
    def device_plane(self, n: int = 1):
        """Zeroed float64 device planes of the library layout, shape (n, nj+2, ld)."""
        import torch
        return torch.zeros((n, self.nj + 2, self.ld), dtype=torch.float64, device=f"cuda:{self.device}")

    def to_device(self, a_ij: np.ndarray):
        """Copy a host [i][j] array into a new device-layout plane."""
        import torch
        src = torch.from_numpy(_as_ij(a_ij, self.ni, self.nj, "array")).to(f"cuda:{self.device}")
        dst = self.device_plane(1)[0]
        s = torch.cuda.current_stream(self.device)
        capi.check(self._L.cth_to_device_layout(self._h, src.data_ptr(), dst.data_ptr(), s.cuda_stream),
                   allow_positive=False)
        s.synchronize()
        return dst

    def to_host(self, plane) -> np.ndarray:
        """Copy a device-layout plane into a new host [i][j] array."""
        import torch
        dst = torch.empty((self.ni + 2, self.nj + 2), dtype=torch.float64, device=f"cuda:{self.device}")
        s = torch.cuda.current_stream(self.device)
        capi.check(self._L.cth_from_device_layout(self._h, plane.data_ptr(), dst.data_ptr(), s.cuda_stream),
                   allow_positive=False)
        s.synchronize()
        return dst.cpu().numpy()

    def smg_solve_dev(self, aP, aE, aW, aN, aS, b, solution, maxITR=30, error_cnv=1e-10,
                      precision=capi.CTH_PREC_FP64, stream=None) -> capi.Status:
        import torch
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        st = capi.Status()
        rc = self._L.cth_smg_solve_dev(self._h, *[_ptr(a) for a in (aP, aE, aW, aN, aS, b)], maxITR,
                                       error_cnv, precision, _ptr(solution), s.cuda_stream, ctypes.byref(st))
        capi.check(rc)
        return st

    def smg_solve_guess_dev(self, aP, aE, aW, aN, aS, b, x0, solution, max_guess_relres=1.0, maxITR=30,
                            error_cnv=1e-10, precision=capi.CTH_PREC_FP64, stream=None) -> capi.Status:
        """smg_solve_dev from the initial guess x0 (a device plane); the guess is
        rejected (zero start) when ||b - A x0|| > max_guess_relres ||b||."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        st = capi.Status()
        rc = self._L.cth_smg_solve_guess_dev(self._h, *[_ptr(a) for a in (aP, aE, aW, aN, aS, b, x0)],
                                             max_guess_relres, maxITR, error_cnv, precision, _ptr(solution),
                                             s.cuda_stream, ctypes.byref(st))
        capi.check(rc)
        return st

    def sor_solve_dev(self, aP, aE, aW, aN, aS, b, solution, alpha_SOR=1.9, maxITR=2000,
                      error_cnv=1e-8, stream=None) -> capi.Status:
        import torch
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        st = capi.Status()
        rc = self._L.cth_sor_solve_dev(self._h, *[_ptr(a) for a in (aP, aE, aW, aN, aS, b)], alpha_SOR,
                                       maxITR, error_cnv, _ptr(solution), s.cuda_stream, ctypes.byref(st))
        capi.check(rc)
        return st

    def residual_dev(self, aP, aE, aW, aN, aS, b, x, r=None, stream=None) -> Tuple[float, float]:
        import torch
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        rn = ctypes.c_double()
        bn = ctypes.c_double()
        capi.check(self._L.cth_residual_dev(self._h, *[_ptr(a) for a in (aP, aE, aW, aN, aS, b, x)],
                                            None if r is None else _ptr(r), ctypes.byref(rn), ctypes.byref(bn),
                                            s.cuda_stream), allow_positive=False)
        return rn.value, bn.value


# grids are reused across calls with the same shape and blocks, as a
# persistent solver would be (the reference rebuilds HYPRE objects per call)
_GRIDS: Dict[tuple, Grid] = {}


def _grid_for(ni, nj, i_bl, j_bl, n_bl, device=0) -> Grid:
    ib = np.asarray(i_bl, dtype=np.int32).reshape(-1, 2)[:n_bl]
    jb = np.asarray(j_bl, dtype=np.int32).reshape(-1, 2)[:n_bl]
    key = (ni, nj, ib.tobytes(), jb.tobytes(), device)
    g = _GRIDS.get(key)
    if g is None:
        g = Grid(ni, nj, ib, jb, n_bl, device)
        _GRIDS[key] = g
    return g


def solver_SMG(aP, aE, aW, aN, aS, b, i_bl, j_bl, n_bl, maxITR, error_cnv, flag_msg, solution,
               precision=capi.CTH_PREC_FP64, device=0) -> capi.Status:
    """solver_SMG (include/solverFuncs.hpp:26-163) on the GPU.

    Zero initial guess; stops when ||b-Ax||_2/||b||_2 < error_cnv or after
    maxITR cycles; writes the grid cells of ``solution`` in place.
    ``flag_msg == 1`` prints the iteration count and final relative residual
    as the reference does (solverFuncs.hpp:131-141).
    """
    ni, nj = solution.shape[0] - 2, solution.shape[1] - 2
    g = _grid_for(ni, nj, i_bl, j_bl, n_bl, device)
    st = g.smg_solve(aP, aE, aW, aN, aS, b, solution, maxITR=maxITR, error_cnv=error_cnv,
                     precision=precision)
    if flag_msg == 1:
        print(f"Number of Iterations: {st.iterations}")
        print(f"Final Relative Residual Norm: {st.residual}")
    return st


def solver_SOR(aP, aE, aW, aN, aS, b, i_bl, j_bl, n_bl, alpha_SOR, maxITR, error_cnv, flag_msg,
               solution, device=0) -> capi.Status:
    """solver_SOR (include/solverFuncs.hpp:169-217) on the GPU, red-black order."""
    ni, nj = solution.shape[0] - 2, solution.shape[1] - 2
    g = _grid_for(ni, nj, i_bl, j_bl, n_bl, device)
    st = g.sor_solve(aP, aE, aW, aN, aS, b, solution, alpha_SOR=alpha_SOR, maxITR=maxITR,
                     error_cnv=error_cnv)
    if flag_msg == 1:
        print(f"ncount = {st.iterations} error_max = {st.residual}")
    return st


class Microwave3:
    """The magnetised 3-component microwave system of solve_Microwave
    (include/emfieldModule.hpp:2249-2998) (cth_mw3): device assembly, the
    coupled operator and the preconditioned BiCGStab solve.  Field planes are
    torch complex128 of shape (3, nj+2, ld): Ex, Er, Ephi in the library layout.

    blocks=None is the r-z rectangle with its walls' boundary lists; otherwise
    blocks = ((xi_bl, xj_bl), (ri_bl, rj_bl), (ci_bl, cj_bl)), the x-face,
    r-face and cell block tables ([n_bl][2] each), and the boundary lists follow
    with set_boundary."""

    NQ = 11
    FIELDS, SIDES = "xrp", "WESN"

    def __init__(self, ni: int, nj: int, device: int = 0, blocks=None):
        L = capi.load()
        h = ctypes.c_void_p()
        if blocks is None:
            capi.check(L.cth_mw3_create(ni, nj, device, ctypes.byref(h)), allow_positive=False)
        else:
            tabs = [np.ascontiguousarray(np.asarray(t, dtype=np.int32).reshape(-1, 2)) for pair in blocks for t in pair]
            args = []
            for f in range(3):
                ib, jb = tabs[2 * f], tabs[2 * f + 1]
                if ib.shape != jb.shape:
                    raise ValueError("i and j block tables of a field differ in length")
                args += [ib.ctypes.data, jb.ctypes.data, ib.shape[0]]
            capi.check(L.cth_mw3_create_blocks(ni, nj, *args, device, ctypes.byref(h)), allow_positive=False)
        self._h, self._L = h, L
        self.ni, self.nj, self.device = ni, nj, device
        self.ld = L.cth_mw3_ld(h)

    def set_boundary(self, lists: dict, j_flc_00: int):
        """lists[(field, side)] = sequence of (i, j, code), field in "xrp" (Ex,
        Er, Ephi), side in "WESN": the 12 lists of MicrowaveBC
        (include/arrays.hpp:649) as makeBoundary builds them; j_flc_00 =
        gc.j_flc_bl[0][0]."""
        keep, arr = [], (capi.BCList * 12)()
        for k, (f, sd) in enumerate((f, sd) for f in self.FIELDS for sd in self.SIDES):
            e = np.asarray(lists.get((f, sd), []), dtype=np.int32).reshape(-1, 3)
            cols = [np.ascontiguousarray(e[:, c]) for c in range(3)]
            keep += cols
            arr[k] = capi.BCList(cols[0].ctypes.data, cols[1].ctypes.data, cols[2].ctypes.data, e.shape[0])
        capi.check(self._L.cth_mw3_set_boundary(self._h, arr, int(j_flc_00)), allow_positive=False)

    def close(self):
        if getattr(self, "_h", None):
            self._L.cth_mw3_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def launch_count(self) -> int:
        return int(self._L.cth_mw3_launch_count(self._h))

    def set_graphs(self, enable: bool):
        """One captured graph per solve (default) or kernel-by-kernel launches."""
        capi.check(self._L.cth_mw3_set_graphs(self._h, int(enable)), allow_positive=False)

    def set_preconditioner(self, mode: int):
        """0: block Jacobi (the fields' V-cycles side by side, default); 1: block
        Gauss-Seidel across Ex, Er, Ephi."""
        capi.check(self._L.cth_mw3_set_preconditioner(self._h, int(mode)), allow_positive=False)

    def set_precision(self, precision: int):
        """CTH_PREC_FP64 (default) or CTH_PREC_MIXED: FP32 complex V-cycles inside the FP64 BiCGStab."""
        capi.check(self._L.cth_mw3_set_precision(self._h, int(precision)), allow_positive=False)

    def set_cycle(self, nu_pre: int, nu_post: int):
        """Smoothing sweeps per level of the three fields' V-cycles (default 1, 1)."""
        capi.check(self._L.cth_mw3_set_cycle(self._h, int(nu_pre), int(nu_post)), allow_positive=False)

    def _stream(self, stream):
        import torch
        return (stream if stream is not None else torch.cuda.current_stream(self.device)).cuda_stream

    def planes(self, n: int = 3):
        import torch
        return torch.zeros((n, self.nj + 2, self.ld), dtype=torch.complex128, device=f"cuda:{self.device}")

    def assemble_dev(self, ne, nu, Bx, Br, epsr, params: dict, stream=None):
        """Assemble from real device planes of cell values (library layout)."""
        prm = capi.MWParams(**{k: float(params[k]) for k, _ in capi.MWParams._fields_})
        capi.check(self._L.cth_mw3_assemble_dev(self._h, _ptr(ne), _ptr(nu), _ptr(Bx), _ptr(Br), _ptr(epsr),
                                                ctypes.byref(prm), self._stream(stream)), allow_positive=False)

    def coefficients(self, stream=None):
        """(a, b): a of shape (3, 11, nj+2, ld), b of shape (3, nj+2, ld)."""
        a = self.planes(3 * self.NQ)
        b = self.planes(3)
        capi.check(self._L.cth_mw3_copy_planes(self._h, _ptr(a), _ptr(b), self._stream(stream)),
                   allow_positive=False)
        return a.reshape(3, self.NQ, self.nj + 2, self.ld), b

    def apply_dev(self, x3, stream=None):
        y = self.planes(3)
        capi.check(self._L.cth_mw3_apply_dev(self._h, _ptr(x3), _ptr(y), self._stream(stream)),
                   allow_positive=False)
        return y

    def fill_ghosts(self, E3, epsr, params: dict, Er_dc=None, stream=None):
        """Ghost values of E3 (in place) from its unknowns, the boundary
        post-processing of solve_Microwave (emfieldModule.hpp:3026-3264);
        Er_dc = gr.Er as a real device plane (needed when the Er east list has
        open entries)."""
        prm = capi.MWParams(**{k: float(params[k]) for k, _ in capi.MWParams._fields_})
        capi.check(self._L.cth_mw3_fill_ghosts(self._h, _ptr(E3), _ptr(epsr),
                                               _ptr(Er_dc) if Er_dc is not None else None, ctypes.byref(prm),
                                               self._stream(stream)), allow_positive=False)

    def solve_dev(self, maxITR: int = 500, error_cnv: float = 1e-10, out=None, stream=None, x0=None,
                  guess_tol: float = 1.0):
        """Returns (E3, status); E3 of shape (3, nj+2, ld), written on the
        unknowns (other entries of `out` keep their values).  x0: an initial
        guess in the same layout (may be `out`), used when its relative residual
        is at most guess_tol (decided on the device), else the zero start."""
        E = out if out is not None else self.planes(3)
        st = capi.Status()
        rc = self._L.cth_mw3_solve_guess_dev(self._h, int(maxITR), float(error_cnv), _ptr(E),
                                             _ptr(x0) if x0 is not None else None, float(guess_tol),
                                             self._stream(stream), ctypes.byref(st))
        capi.check(rc)
        return E, st
