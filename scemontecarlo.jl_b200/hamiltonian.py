"""Host-side table builder: the tiled SCE Hamiltonian in the reference's flat layout.

`TiledHamiltonian` mirrors src/hamiltonian.jl:234-393 (constructor), its programs
(62-181), the Zeeman templates (405-448) and the greedy colouring (456-499), with
the same 1-based arrays, entry order and skip predicates, so the tables it hands
to libscemc_cuda.so are the ones a Julia caller would pass from its own
`TiledHamiltonian`. The instance enumeration and the CSR are vectorised with
numpy; the greedy colouring (inherently sequential) runs in the library's host
helper `scemc_color_sites`.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib

FOUR_PI = 12.566370614359172            # Float64(4π)
KB_EV = 1.380649e-23 / 1.602176634e-19  # src/units.jl:17
MU_B_EV_T = 9.2740100783e-24 / 1.602176634e-19  # src/units.jl:29
N1 = math.sqrt(3.0 / FOUR_PI)           # Z_1m = N1 * (y, z, x)


@dataclass
class MultipoleTerm:
    """One raw (unscaled) SCE term, the SCEFitting `MultipoleTerm` fields the tiling
    reads: coefficient, member atoms (1-based, training cell), per-member lattice
    shifts (shifts[0] == (0,0,0)), per-member angular momenta, and the dense
    coefficient tensor `folded` of shape (2l_1+1, ..., 2l_b+1)."""

    coef: float
    atoms: Sequence[int]
    shifts: Sequence[Sequence[int]]
    ls: Sequence[int]
    folded: np.ndarray

    @property
    def body(self) -> int:
        return len(self.atoms)


@dataclass
class ScaledTerm:
    coef: float
    atoms: list
    shifts: np.ndarray  # (body, 3) int
    ls: list
    folded: np.ndarray  # column-major flattened


def _lm0(l: int, m: int) -> int:
    return l * l + l + m


def resolve_kt(temperature=None, kT=None) -> np.ndarray:
    """src/units.jl:40-61: exactly one of kelvin `temperature` or `kT`."""
    if (temperature is None) == (kT is None):
        raise ValueError("provide exactly one of `temperature` (kelvin) or `kT` (k_B·T, model energy units)")
    if kT is not None:
        vals = np.atleast_1d(np.asarray(kT, dtype=np.float64))
    else:
        ts = np.atleast_1d(np.asarray(temperature, dtype=np.float64))
        for T in ts:
            if not (np.isfinite(T) and T > 0):
                raise ValueError(f"temperature must be finite and > 0 kelvin; got {T}")
        vals = KB_EV * ts
    if vals.size == 0:
        raise ValueError("the temperature/kT collection is empty")
    for x in vals:
        if not (np.isfinite(x) and x > 0):
            raise ValueError(f"kT must be finite and > 0 (k_B·T, model energy units); got {x}")
    return vals


class TiledHamiltonian:
    """The fitted SCE Hamiltonian tiled onto an N1 x N2 x N3 supercell.

    Attributes follow the reference struct (src/hamiltonian.jl:234-265); the
    program arrays live in `self.progs` as plain numpy arrays (1-based indices).
    """

    def __init__(self, n_cell_atoms: int, terms: Sequence[MultipoleTerm], dims=(1, 1, 1),
                 magmoms: Optional[Sequence[float]] = None, field=None):
        if n_cell_atoms < 1:
            raise ValueError(f"n_cell_atoms must be ≥ 1; got {n_cell_atoms}")
        d = np.asarray(dims, dtype=np.int64)
        if d.shape != (3,) or np.any(d < 1):
            raise ValueError(f"dims must be ≥ 1; got {dims}")
        self.n_cell_atoms = int(n_cell_atoms)
        self.dims = tuple(int(x) for x in d)
        mm, B = self._resolve_zeeman(magmoms, field)
        self.magmoms = mm
        self.field = B
        zterms = self._zeeman_terms(mm, B)
        mterms = [t for t in terms if t.coef != 0.0]
        if not mterms and not zterms:
            raise ValueError("the term list is empty (no spin-dependent SALCs with nonzero coefficients "
                             "and no Zeeman term)")
        scaled = []
        lmax = 0
        for k, mt in enumerate(mterms):
            body = len(mt.atoms)
            if len(mt.shifts) != body or len(mt.ls) != body:
                raise ValueError(f"term {k + 1}: atoms/shifts/ls lengths disagree")
            if any(not (1 <= a <= n_cell_atoms) for a in mt.atoms):
                raise ValueError(f"term {k + 1}: atoms {list(mt.atoms)} outside 1:{n_cell_atoms}")
            sh = np.asarray(mt.shifts, dtype=np.int64).reshape(body, 3)
            keys = {(int(a), *(int(x) for x in np.mod(s, d))) for a, s in zip(mt.atoms, sh)}
            if len(keys) != body:
                raise ValueError(f"term {k + 1} folds two member sites onto one supercell site under "
                                 f"dims = {self.dims}; enlarge dims")
            if np.any(sh[0] != 0):
                raise ValueError(f"term {k + 1}: shifts[1] must be zero (home-cell anchoring)")
            if any(l < 0 for l in mt.ls):
                raise ValueError(f"term {k + 1}: negative angular momentum in {list(mt.ls)}")
            f = np.asarray(mt.folded, dtype=np.float64)
            if f.shape != tuple(2 * l + 1 for l in mt.ls):
                raise ValueError(f"term {k + 1}: size(folded) = {f.shape} does not match ls = {list(mt.ls)}")
            lmax = max(lmax, max(mt.ls))
            scaled.append(ScaledTerm(mt.coef * math.pow(FOUR_PI, body / 2.0), [int(a) for a in mt.atoms],
                                     sh, [int(l) for l in mt.ls], f.ravel(order="F").copy()))
        self.n_fitted_terms = len(scaled)
        if zterms:
            scaled = scaled + zterms
            lmax = max(lmax, 1)
        self.terms = scaled
        self.lmax = lmax
        self.nlm = (lmax + 1) ** 2
        d1, d2, d3 = self.dims
        ncells = d1 * d2 * d3
        self.n_sites = n_cell_atoms * ncells
        self._tile(d)
        self._build_programs()
        self._color()

    # -- Zeeman (hamiltonian.jl:405-448)
    def _resolve_zeeman(self, magmoms, field):
        mm = None
        if magmoms is not None:
            mm = np.asarray(magmoms, dtype=np.float64).ravel()
            if mm.size != self.n_cell_atoms:
                raise ValueError(f"magmoms has {mm.size} entries but the cell has {self.n_cell_atoms} atoms")
            if not np.all(np.isfinite(mm) & (mm >= 0)):
                raise ValueError(f"magmoms must be finite and ≥ 0; got {mm}")
        B = np.zeros(3)
        if field is not None:
            if mm is None:
                raise ValueError("field given without magmoms: the Zeeman energy needs moment magnitudes")
            B = np.asarray(field, dtype=np.float64).ravel()
            if B.size != 3:
                raise ValueError("field must have 3 components (tesla)")
            if not np.all(np.isfinite(B)):
                raise ValueError("field must be finite (tesla)")
        return mm, B

    @staticmethod
    def _zeeman_terms(mm, B):
        out = []
        if mm is None or not np.any(B != 0):
            return out
        for a, m in enumerate(mm):
            if m == 0.0:
                continue
            sc = -(MU_B_EV_T * m / N1)
            hz = np.array([sc * B[1], sc * B[2], sc * B[0]])
            out.append(ScaledTerm(1.0, [a + 1], np.zeros((1, 3), dtype=np.int64), [1], hz))
        return out

    def has_field(self) -> bool:
        return bool(np.any(self.field != 0))

    # -- instances + per-site CSR (hamiltonian.jl:333-383)
    def _tile(self, d):
        d1, d2, d3 = self.dims
        ncells = d1 * d2 * d3
        nca = self.n_cell_atoms
        cell = np.arange(ncells, dtype=np.int64)
        c1, c2, c3 = cell % d1, (cell // d1) % d2, cell // (d1 * d2)
        bodies = np.array([len(t.atoms) for t in self.terms], dtype=np.int64)
        cols = []
        for t in self.terms:
            for a, sh in zip(t.atoms, t.shifts):
                w1 = np.mod(c1 + sh[0], d1)
                w2 = np.mod(c2 + sh[1], d2)
                w3 = np.mod(c3 + sh[2], d3)
                cols.append(a + nca * (w1 + d1 * (w2 + d2 * w3)))
        per_cell = int(bodies.sum())
        inst_sites = np.stack(cols, axis=1).reshape(-1) if cols else np.zeros(0, np.int64)
        nterms = len(self.terms)
        n_inst = nterms * ncells
        inst_body = np.tile(bodies, ncells)
        self.inst_term = np.tile(np.arange(1, nterms + 1, dtype=np.int32), ncells)
        self.inst_ptr = np.concatenate([[1], 1 + np.cumsum(inst_body)]).astype(np.int32)
        self.inst_sites = inst_sites.astype(np.int32)
        counts = np.bincount(inst_sites - 1, minlength=self.n_sites)
        self.site_ptr = np.concatenate([[1], 1 + np.cumsum(counts)]).astype(np.int32)
        order = np.argsort(inst_sites, kind="stable")
        entry_inst = np.repeat(np.arange(1, n_inst + 1, dtype=np.int64), inst_body)
        slot_pattern = np.concatenate([np.arange(1, b + 1) for b in bodies])
        entry_slot = np.tile(slot_pattern, ncells)
        self.site_inst = entry_inst[order].astype(np.int32)
        self.site_slot = entry_slot[order].astype(np.int8)
        ls_pattern = np.concatenate([np.asarray(t.ls) for t in self.terms])
        entry_l1 = np.tile(ls_pattern == 1, ncells)
        self.site_has_l1 = (np.bincount(inst_sites - 1, weights=entry_l1, minlength=self.n_sites) > 0)
        self.site_active = counts > 0
        self.n_active = int(self.site_active.sum())
        if int(per_cell) * ncells >= 2 ** 31:
            raise ValueError("model too large for Int32 tables")

    # -- programs (hamiltonian.jl:99-181)
    def _build_programs(self):
        sent_w, sent_tgt, sfac_ptr, sfac_row, sfac_slot = [], [], [1], [], []
        pent_row, pent_row2, sprog_ptr = [], [], [1]
        eent_w, efac_ptr, efac_row, eprog_ptr = [], [1], [], [1]
        pbase, pslot1, pslot2 = [], [], []
        np_ = 0
        for t in self.terms:
            D = len(t.ls)
            pbase.append(np_)
            np_ += D
            for v in range(1, D + 1):
                pslot1.append((3 - v) if D == 2 else ((2 if v == 1 else 1) if D == 3 else 0))
                pslot2.append((2 if v == 3 else 3) if D == 3 else 0)
            dims = [2 * l + 1 for l in t.ls]
            idxs = list(np.ndindex(*dims[::-1]))  # C order over reversed dims == column-major
            idxs = [ix[::-1] for ix in idxs]
            for v in range(D):
                for lin, ix in enumerate(idxs):
                    w = t.coef * t.folded[lin]
                    if w == 0.0:
                        continue
                    sent_w.append(w)
                    sent_tgt.append(_lm0(t.ls[v], ix[v] - t.ls[v]) + 1)
                    for k in range(D):
                        if k == v:
                            continue
                        sfac_row.append(_lm0(t.ls[k], ix[k] - t.ls[k]) + 1)
                        sfac_slot.append(k + 1)
                    sfac_ptr.append(len(sfac_row) + 1)
                    pent_row.append(sfac_row[-1] if D == 2 else (sfac_row[-2] if D == 3 else 0))
                    pent_row2.append(sfac_row[-1] if D == 3 else 0)
                sprog_ptr.append(len(sent_w) + 1)
            for lin, ix in enumerate(idxs):
                w = t.folded[lin]
                if w == 0.0:
                    continue
                eent_w.append(w)
                for k in range(D):
                    efac_row.append(_lm0(t.ls[k], ix[k] - t.ls[k]) + 1)
                efac_ptr.append(len(efac_row) + 1)
            eprog_ptr.append(len(eent_w) + 1)
        i32 = lambda x: np.asarray(x, dtype=np.int32)
        self.sent_w = np.asarray(sent_w, dtype=np.float64)
        self.sent_tgt = i32(sent_tgt)
        self.sfac_ptr = i32(sfac_ptr)
        self.sfac_row = i32(sfac_row)
        self.sfac_slot = np.asarray(sfac_slot, dtype=np.int8)
        self.pent_row = i32(pent_row)
        self.pent_row2 = i32(pent_row2)
        self.sprog_ptr = i32(sprog_ptr)
        self.eent_w = np.asarray(eent_w, dtype=np.float64)
        self.efac_ptr = i32(efac_ptr)
        self.efac_row = i32(efac_row)
        self.eprog_ptr = i32(eprog_ptr)
        self.term_coef = np.asarray([t.coef for t in self.terms], dtype=np.float64)
        self.term_body = i32([len(t.ls) for t in self.terms])
        self.term_ls = i32([l for t in self.terms for l in t.ls])
        pbase = np.asarray(pbase, dtype=np.int64)
        pslot1 = np.asarray(pslot1, dtype=np.int64)
        pslot2 = np.asarray(pslot2, dtype=np.int64)
        inst = self.site_inst.astype(np.int64)
        pid = pbase[self.inst_term[inst - 1] - 1] + self.site_slot.astype(np.int64)
        self.site_prog = pid.astype(np.int32)
        off = self.inst_ptr[inst - 1].astype(np.int64) - 1
        sl1 = pslot1[pid - 1]
        sl2 = pslot2[pid - 1]
        col1 = self.inst_sites[np.where(sl1 > 0, off + sl1 - 1, 0)]
        col2 = self.inst_sites[np.where(sl2 > 0, off + sl2 - 1, 0)]
        self.site_col = np.where(sl1 == 0, 0, np.where(sl2 == 0, col1, -col1)).astype(np.int32)
        self.site_col2 = np.where(sl2 == 0, 0, col2).astype(np.int32)

    # -- greedy colouring (hamiltonian.jl:456-499) through the library helper
    def _color(self):
        L = _lib.lib()
        colors = np.zeros(self.n_sites, dtype=np.int32)
        ncol = C.c_int32(0)
        active = self.site_active.astype(np.uint8)
        _lib.check(L.scemc_color_sites(self.n_sites, _lib.ptr(self.site_ptr, C.c_int32),
                                       _lib.ptr(self.site_inst, C.c_int32), _lib.ptr(self.inst_ptr, C.c_int32),
                                       _lib.ptr(self.inst_sites, C.c_int32), _lib.ptr(active, C.c_uint8),
                                       _lib.ptr(colors, C.c_int32), C.byref(ncol)))
        n = ncol.value
        counts = np.bincount(colors, minlength=n + 1)[1:]
        self.n_colors = n
        self.color_ptr = np.concatenate([[1], 1 + np.cumsum(counts)]).astype(np.int32)
        sites = np.arange(1, self.n_sites + 1, dtype=np.int32)
        order = np.argsort(colors, kind="stable")
        self.color_sites = sites[order][colors[order] > 0].astype(np.int32)
        self.colors = colors

    # -- helpers
    def site_atom(self, s: int) -> int:
        """Training-cell atom (sublattice) of 1-based site s (hamiltonian.jl:549)."""
        return (int(s) - 1) % self.n_cell_atoms + 1

    def site_index(self, atom: int, cell) -> int:
        c = [int(x) for x in cell]
        d1, d2, _ = self.dims
        return atom + self.n_cell_atoms * (c[0] + d1 * (c[1] + d2 * c[2]))

    def arrays(self) -> dict:
        """The flat tables by reference name (1-based)."""
        names = ["inst_term", "inst_ptr", "inst_sites", "site_ptr", "site_inst", "site_slot", "site_prog",
                 "sprog_ptr", "sent_w", "sent_tgt", "sfac_ptr", "sfac_row", "sfac_slot", "site_col", "site_col2",
                 "pent_row", "pent_row2", "eprog_ptr", "eent_w", "efac_ptr", "efac_row", "term_coef",
                 "color_ptr", "color_sites"]
        out = {n: getattr(self, n) for n in names}
        out["site_has_l1"] = self.site_has_l1.astype(np.uint8)
        out["site_active"] = self.site_active.astype(np.uint8)
        return out

    def desc(self):
        """A `scemc_tables_desc` over this object's arrays (kept alive by `self`)."""
        keep = {}

        def arr(name, dtype):
            a = np.ascontiguousarray(getattr(self, name), dtype=dtype)
            keep[name] = a
            return a

        d = _lib.TablesDesc()
        d.n_sites, d.nlm, d.lmax, d.n_colors = self.n_sites, self.nlm, self.lmax, self.n_colors
        d.n_active, d.n_cell_atoms = self.n_active, self.n_cell_atoms
        d.n_adj = len(self.site_inst)
        d.n_inst = len(self.inst_term)
        d.n_inst_sites = len(self.inst_sites)
        d.n_sprog = len(self.sprog_ptr) - 1
        d.n_sent = len(self.sent_w)
        d.n_sfac = len(self.sfac_row)
        d.n_terms = len(self.terms)
        d.n_eent = len(self.eent_w)
        d.n_efac = len(self.efac_row)
        for name in ["site_ptr", "site_inst", "inst_term", "inst_ptr", "inst_sites", "site_prog", "sprog_ptr",
                     "sent_tgt", "sfac_ptr", "sfac_row", "site_col", "site_col2", "pent_row", "pent_row2",
                     "eprog_ptr", "efac_ptr", "efac_row", "term_body", "term_ls", "color_ptr", "color_sites"]:
            setattr(d, name, _lib.ptr(arr(name, np.int32), C.c_int32))
        for name in ["site_slot", "sfac_slot"]:
            setattr(d, name, _lib.ptr(arr(name, np.int8), C.c_int8))
        for name in ["sent_w", "eent_w", "term_coef"]:
            setattr(d, name, _lib.ptr(arr(name, np.float64), C.c_double))
        for name in ["site_has_l1", "site_active"]:
            setattr(d, name, _lib.ptr(arr(name, np.uint8), C.c_uint8))
        d._keep = keep
        return d

    def __repr__(self):
        nz = len(self.terms) - self.n_fitted_terms
        return (f"TiledHamiltonian({self.n_cell_atoms} atoms × {self.dims[0]}×{self.dims[1]}×{self.dims[2]} = "
                f"{self.n_sites} sites, lmax={self.lmax}, "
                + (f"{len(self.terms)} terms" if nz == 0 else f"{self.n_fitted_terms} fitted + {nz} zeeman terms")
                + f", {len(self.inst_term)} instances)")
