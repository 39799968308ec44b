"""Python face of libbsgpu.so (the sm_100a engine).

Mirrors the reference's operator interface for this path:

* ``Hamiltonian(tables)``        -- bsg_create: validate + upload the tables
* ``H.applyh(vin, vout=None, accumulate=False)``
                                 -- applyHbundled_omp('n') / applyHbundled_block_omp:
                                    vout (+)= H vin, nb inferred from the shape
                                    (dim,) or (dim, nb) (interleaved layout)
* ``H.lanczos(...)``             -- lanczos_p / lanczos_block with thick restart
* ``H.grad(evecs)``              -- adjoint: dE/dhmat for every uncoupled label
* ``H.density1b(vecs)``          -- master_density1b_bundled for every state pair
* ``H.apply1b(ppot, npot, v)``   -- master_apply1bop: a one-body operator on vectors

Errors raise ``BsgError`` with the status name and the latched message; there
is no CPU fallback anywhere on this path.
"""
import ctypes as C
import json
import os

import numpy as np

from . import _abi


class BsgError(RuntimeError):
    def __init__(self, status, msg):
        self.status = status
        super().__init__(f"{_abi.STATUS_NAMES.get(status, status)}: {msg}")


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def validate_tables(tables):
    """Run bsg_create's table validator on the host (no GPU needed).
    Returns (status, message); status 0 means valid."""
    lib = _abi.gpu_lib()
    t = tables.as_ctypes()
    buf = C.create_string_buffer(512)
    t3 = tables.as_ctypes3() if getattr(tables, "threebody", False) else None
    if t3 is not None:
        st = lib.bsg_validate_tables3(C.byref(t), C.byref(t3), buf, 512)
    else:
        st = lib.bsg_validate_tables(C.byref(t), buf, 512)
    return st, buf.value.decode()


class Hamiltonian:
    def __init__(self, tables, device=0, max_nb=16, validate=True, pn_table_max=0):
        """pn_table_max: largest (b,d) table of one neutron operator before
        it is split into sub-operators (bsg_config.pn_table_max; 0 = 512, or
        384 for a three-body Hamiltonian)."""
        self.lib = _abi.gpu_lib()
        self.tables = tables
        self._ct = tables.as_ctypes()
        cfg = _abi.BsgConfig(device, max_nb, 1 if validate else 0, int(pn_table_max))
        h = C.c_void_p()
        # a three-body Hamiltonian (model.build_tables3) goes through bsg_create3
        self._ct3 = tables.as_ctypes3() if getattr(tables, "threebody", False) else None
        if self._ct3 is not None:
            st = self.lib.bsg_create3(C.byref(self._ct), C.byref(self._ct3), C.byref(cfg), C.byref(h))
        else:
            st = self.lib.bsg_create(C.byref(self._ct), C.byref(cfg), C.byref(h))
        if st != 0:
            raise BsgError(st, "bsg_create failed (see stderr for the validator message)")
        self.h = h
        self.dim = tables.dim

    def close(self):
        if getattr(self, "h", None):
            self.lib.bsg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st != 0:
            buf = C.create_string_buffer(512)
            self.lib.bsg_last_error(self.h, buf, 512)
            raise BsgError(st, f"{what}: {buf.value.decode()}")

    def stats(self):
        s = _abi.BsgStats()
        self._check(self.lib.bsg_get_stats(self.h, C.byref(s)), "bsg_get_stats")
        return {k: getattr(s, k) for k, _ in s._fields_}

    # ------------------------------------------------------------ applyH
    def applyh(self, vin, vout=None, accumulate=False, stream=None):
        """vout (+)= H vin.  numpy arrays use host pointers (copies inside the
        call); torch CUDA tensors use device pointers on the current stream."""
        nb = 1 if vin.ndim == 1 else int(vin.shape[1])
        if vin.shape[0] != self.dim:
            raise ValueError(f"vector length {vin.shape[0]} != dim {self.dim}")
        if _is_torch(vin):
            import torch
            prec = 4 if vin.dtype == torch.float32 else 8
            if vin.dtype not in (torch.float32, torch.float64) or not vin.is_cuda or not vin.is_contiguous():
                raise ValueError("torch input must be a contiguous CUDA float32/float64 tensor")
            if vout is None:
                vout = torch.empty_like(vin)
            flags = _abi.BSG_DEVICE_PTRS | (_abi.BSG_ACCUMULATE if accumulate else 0)
            s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
            st = self.lib.bsg_applyh_stream(self.h, C.c_void_p(vin.data_ptr()), C.c_void_p(vout.data_ptr()),
                                            nb, prec, flags, C.c_void_p(s))
            self._check(st, "bsg_applyh")
            return vout
        vin = np.ascontiguousarray(vin)
        if vin.dtype not in (np.float32, np.float64):
            raise ValueError("vector dtype must be float32 or float64")
        prec = 4 if vin.dtype == np.float32 else 8
        if vout is None:
            vout = np.zeros_like(vin)
        flags = _abi.BSG_ACCUMULATE if accumulate else 0
        st = self.lib.bsg_applyh(self.h, vin.ctypes.data, vout.ctypes.data, nb, prec, flags)
        self._check(st, "bsg_applyh")
        return vout

    # ----------------------------------------------------------- Lanczos
    def lanczos(self, nkeep=10, niter=300, nthick_add=0, max_restarts=0, nb=1, matvec_prec=8,
                fixed_iter=False, ncheck=None, converge_tol=1e-3, want_vectors=False, pivot=None,
                seed=12345, lanc_prec=8):
        """lanczos_p (nb = 1) / lanczos_block (nb > 1) with thick restart.
        matvec_prec: applyH precision (4 or 8); lanc_prec: storage of the
        Lanczos vectors (4 or 8, the reference's lanc_prec), dots and updates
        accumulating in FP64 either way.  Returns (eigenvalues, eigenvectors
        dim x nkeep or None, report dict)."""
        p = _abi.BsgLanczosParams()
        p.nkeep = nkeep
        p.niter = niter
        p.nthick_add = nthick_add
        p.max_restarts = max_restarts
        p.nb = nb
        p.matvec_prec = matvec_prec
        p.fixed_iter = 1 if fixed_iter else 0
        p.ncheck = ncheck if ncheck is not None else nkeep + 5
        p.converge_tol = converge_tol
        p.want_vectors = 1 if want_vectors else 0
        p.pivot = 0
        p.seed = seed
        p.lanc_prec = lanc_prec
        ev = np.zeros(nkeep, dtype=np.float64)
        vecs = np.zeros((nkeep, self.dim), dtype=np.float64) if want_vectors else None
        pv = None
        if pivot is not None:
            pv = np.ascontiguousarray(pivot, dtype=np.float64)
            if pv.size != self.dim * nb:
                raise ValueError("pivot must have dim*nb entries")
        rep = _abi.BsgReport()
        st = self.lib.bsg_lanczos(self.h, C.byref(p),
                                  pv.ctypes.data_as(_abi.f64p) if pv is not None else None,
                                  ev.ctypes.data_as(_abi.f64p),
                                  vecs.ctypes.data_as(_abi.f64p) if vecs is not None else None,
                                  C.byref(rep))
        self._check(st, "bsg_lanczos")
        report = {k: getattr(rep, k) for k, _ in rep._fields_}
        return ev, (vecs.T.copy() if vecs is not None else None), report

    # ----------------------------------------------------------- adjoint
    def grad(self, evecs):
        """dE_k/dhmat for each state k: dict of (nstates, nmat) arrays for
        'pp', 'nn', 'pn' (and 'spe_p', 'spe_n' when call_spe)."""
        ev = np.ascontiguousarray(np.asarray(evecs, dtype=np.float64).T)  # (nstates, dim)
        ns = ev.shape[0]
        s = self.tables.s
        out = {"pp": np.zeros((ns, s["nmatpp"])), "nn": np.zeros((ns, s["nmatnn"])),
               "pn": np.zeros((ns, s["nmatpn"]))}
        sp = sn = None
        if s["call_spe"]:
            out["spe_p"] = np.zeros((ns, s["nsd_p"]))
            out["spe_n"] = np.zeros((ns, s["nsd_n"]))
            sp, sn = out["spe_p"], out["spe_n"]
        st = self.lib.bsg_grad(self.h, ev.ctypes.data_as(_abi.f64p), ns,
                               out["pp"].ctypes.data_as(_abi.f64p), out["nn"].ctypes.data_as(_abi.f64p),
                               out["pn"].ctypes.data_as(_abi.f64p),
                               sp.ctypes.data_as(_abi.f64p) if sp is not None else None,
                               sn.ctypes.data_as(_abi.f64p) if sn is not None else None)
        self._check(st, "bsg_grad")
        return out

    def density1b(self, vecs, density_tables=None):
        """m-scheme one-body transition densities of every pair of the states
        `vecs` (dim x k; above 32 states the pairs are computed in tiles of
        two 16-state blocks, bsg_density1b taking 32 at most): {'p': D_p,
        'n': D_n} with
        D[f, i, c, d] = <f| a+_c a_d |i>, c and d the combined s.p. indices of
        the builder (``extra['sp_orb_p']`` etc.).  `density_tables`: a
        ``bsg_density_tables`` (default: the builder's own, from these
        tables)."""
        v = np.asarray(vecs, dtype=np.float64)
        if v.ndim == 1:
            v = v[:, None]
        if v.shape[0] != self.dim:
            raise ValueError("vectors do not match the basis")
        if v.shape[1] > 32:
            from .densities import tiled_pairs
            return tiled_pairs(v.shape[1], lambda idx: self.density1b(v[:, idx], density_tables))
        cols = np.ascontiguousarray(v.T)  # (k, dim): dim x k column-major
        ns = cols.shape[0]
        s = self.tables.s
        nqp = int(s["nhsps_pl"] + s["nhsps_pr"])
        nqn = int(s["nhsps_nl"] + s["nhsps_nr"])
        dp = np.zeros((ns, ns, nqp, nqp))
        dn = np.zeros((ns, ns, nqn, nqn))
        dt = density_tables if density_tables is not None else self.tables.density_ctypes()
        st = self.lib.bsg_density1b(self.h, C.byref(dt), cols.ctypes.data_as(_abi.f64p), ns,
                                    dp.ctypes.data_as(_abi.f64p), dn.ctypes.data_as(_abi.f64p))
        self._check(st, "bsg_density1b")
        return {"p": dp, "n": dn}

    def apply1b(self, ppot, npot, vecs, density_tables=None):
        """O v for the one-body operator O = sum_cd ppot[c, d] a+_c a_d
        (protons) + npot[c, d] a+_c a_d (neutrons) on the combined s.p.
        indices (None: no such part); vecs: dim or dim x k.  Returns the same
        shape."""
        v = np.asarray(vecs, dtype=np.float64)
        one = v.ndim == 1
        if one:
            v = v[:, None]
        if v.shape[0] != self.dim:
            raise ValueError("vectors do not match the basis")
        cols = np.ascontiguousarray(v.T)
        out = np.zeros_like(cols)
        pp = None if ppot is None else np.ascontiguousarray(ppot, dtype=np.float64)
        nn = None if npot is None else np.ascontiguousarray(npot, dtype=np.float64)
        dt = density_tables if density_tables is not None else self.tables.density_ctypes()
        st = self.lib.bsg_apply1b(self.h, C.byref(dt), pp.ctypes.data_as(_abi.f64p) if pp is not None else None,
                                  nn.ctypes.data_as(_abi.f64p) if nn is not None else None,
                                  cols.ctypes.data_as(_abi.f64p), out.ctypes.data_as(_abi.f64p), cols.shape[0])
        self._check(st, "bsg_apply1b")
        return out[0] if one else out.T


def angular_momentum_isospin(spec, vecs, device=0):
    """J and T of the states `vecs` (dim x k, columns normalized, in the basis
    of `spec`): <J^2> and <T^2> with the operators of model.jsq_spec /
    model.tsq_spec applied by the engine in FP64, as lanczos_output reports
    them.  Returns (J, T) arrays."""
    from . import model
    v = np.ascontiguousarray(np.asarray(vecs, dtype=np.float64))
    if v.ndim == 1:
        v = v[:, None]
    out = []
    for mk in (model.jsq_spec, model.tsq_spec):
        T = model.build_tables(mk(spec))
        if T.dim != v.shape[0]:
            raise ValueError("vectors do not match the basis of the model")
        H = Hamiltonian(T, device=device)
        try:
            ex = np.array([float(v[:, k] @ H.applyh(np.ascontiguousarray(v[:, k]))) for k in range(v.shape[1])])
        finally:
            H.close()
        out.append(model.j_from_jsq(ex))
    return out[0], out[1]


class _SystemView(Hamiltonian):
    """A Hamiltonian bound to one system of a Batch (the batch owns it)."""

    def __init__(self, lib, handle, tables):
        self.lib = lib
        self.tables = tables
        self.h = handle
        self.dim = tables.dim

    def close(self):
        self.h = None


class Batch:
    """Many independent Hamiltonians (bsg_batch_*): one persistent launch
    applies all of them; Lanczos runs lock-step with one captured CUDA graph
    per iteration.

    tune_cache: JSON file mapping a batch signature to the autotuned
    (tile width, CTAs per SM); read if present, written after autotuning."""

    def __init__(self, tables_list, device=0, autotune=False, tune_cache=None):
        self.lib = _abi.gpu_lib()
        self.tables = list(tables_list)
        self._ct = [t.as_ctypes() for t in self.tables]
        arr = (C.POINTER(_abi.BsgTables) * len(self._ct))(*[C.pointer(t) for t in self._ct])
        cfg = _abi.BsgConfig(device, 16, 1, 0)
        h = C.c_void_p()
        st = self.lib.bsg_batch_create(len(self._ct), arr, C.byref(cfg), C.byref(h))
        if st != 0:
            raise BsgError(st, "bsg_batch_create failed")
        self.h = h
        self.dims = [t.dim for t in self.tables]
        self.tuning = None
        sig = self.signature()
        cache = {}
        if tune_cache:
            if os.path.exists(tune_cache):
                cache = json.load(open(tune_cache))
        if sig in cache:
            items, ctas = cache[sig]["items"], cache[sig]["ctas_per_sm"]
            self._check(self.lib.bsg_batch_set_tuning(self.h, items, ctas), "bsg_batch_set_tuning")
            self.tuning = dict(cache[sig], source="cache")
        elif autotune:
            self.tuning = self.autotune()
            if tune_cache:
                cache[sig] = {k: v for k, v in self.tuning.items() if k != "source"}
                os.makedirs(os.path.dirname(os.path.abspath(tune_cache)), exist_ok=True)
                with open(tune_cache, "w") as f:
                    json.dump(cache, f, indent=1)

    def signature(self):
        import hashlib
        h = hashlib.sha256()
        for t in self.tables:
            h.update(str((t.dim, t.s["np1b"], t.s["np2b"], t.s["nn1b"], t.s["nn2b"])).encode())
        return h.hexdigest()[:16]

    def _check(self, st, what):
        if st != 0:
            buf = C.create_string_buffer(512)
            self.lib.bsg_batch_last_error(self.h, buf, 512)
            raise BsgError(st, f"{what}: {buf.value.decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.bsg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def system(self, s):
        ctx = C.c_void_p()
        self._check(self.lib.bsg_batch_system(self.h, s, C.byref(ctx)), "bsg_batch_system")
        return _SystemView(self.lib, ctx, self.tables[s])

    def autotune(self):
        it, cps, ms = C.c_int(), C.c_int(), C.c_double()
        self._check(self.lib.bsg_batch_autotune(self.h, C.byref(it), C.byref(cps), C.byref(ms)), "autotune")
        return {"items": it.value, "ctas_per_sm": cps.value, "ms": ms.value, "source": "autotune"}

    def applyh(self, vins, vouts, stream=None):
        """vins/vouts: lists of contiguous CUDA tensors (float32 or float64)."""
        import torch
        prec = 4 if vins[0].dtype == torch.float32 else 8
        vi = (C.c_void_p * len(vins))(*[v.data_ptr() for v in vins])
        vo = (C.c_void_p * len(vouts))(*[v.data_ptr() for v in vouts])
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        self._check(self.lib.bsg_batch_applyh(self.h, vi, vo, prec, C.c_void_p(s)), "bsg_batch_applyh")

    def grad(self, vecs):
        """Adjoint gradients of every system in one launch (bsg_batch_grad):
        vecs[s] dim_s x k eigenvectors of system s; returns a list of dicts
        of (k, nmat) arrays 'pp', 'nn', 'pn' (and 'spe_p', 'spe_n' for
        members with SPE bundles), bitwise equal to each member's own
        Hamiltonian.grad, and sets self.grad_ms to the launch's device time."""
        n = len(self.tables)
        if len(vecs) != n:
            raise ValueError("one eigenvector block per system")
        k = np.asarray(vecs[0]).shape[1] if np.asarray(vecs[0]).ndim == 2 else 1
        cols, outs = [], []
        for t, v in zip(self.tables, vecs):
            v = np.asarray(v, dtype=np.float64).reshape(t.dim, -1)
            if v.shape[1] != k:
                raise ValueError("every system needs the same number of states")
            cols.append(np.ascontiguousarray(v.T))
            s = t.s
            o = {"pp": np.zeros((k, s["nmatpp"])), "nn": np.zeros((k, s["nmatnn"])), "pn": np.zeros((k, s["nmatpn"]))}
            if s["call_spe"]:
                o["spe_p"] = np.zeros((k, s["nsd_p"]))
                o["spe_n"] = np.zeros((k, s["nsd_n"]))
            outs.append(o)
        arr = lambda xs: (_abi.f64p * n)(*[x.ctypes.data_as(_abi.f64p) if x is not None else None for x in xs])
        ms = C.c_double()
        st = self.lib.bsg_batch_grad(self.h, arr(cols), k, arr([o["pp"] for o in outs]), arr([o["nn"] for o in outs]),
                                     arr([o["pn"] for o in outs]), arr([o.get("spe_p") for o in outs]),
                                     arr([o.get("spe_n") for o in outs]), C.byref(ms))
        self._check(st, "bsg_batch_grad")
        self.grad_ms = ms.value
        return outs

    def lanczos(self, nkeep=5, niter=150, matvec_prec=8, want_vectors=False, pivot="uniform", seed=12345):
        """Lock-step Lanczos over all systems, exactly niter iterations.
        pivot: "uniform" (the reference's option 0) or "random" (a seeded
        random normalized pivot per system)."""
        p = _abi.BsgLanczosParams()
        p.nkeep, p.niter, p.nb, p.matvec_prec, p.fixed_iter = nkeep, niter, 1, matvec_prec, 1
        if pivot not in ("uniform", "random"):
            raise ValueError("pivot must be 'uniform' or 'random'")
        p.pivot = 1 if pivot == "random" else 0
        p.seed = seed
        ev = np.zeros(len(self.tables) * nkeep)
        vecs = [np.zeros((nkeep, d)) for d in self.dims] if want_vectors else None
        vp = (_abi.f64p * len(self.tables))(*[v.ctypes.data_as(_abi.f64p) for v in vecs]) if vecs else None
        rep = _abi.BsgReport()
        self._check(self.lib.bsg_batch_lanczos(self.h, C.byref(p), ev.ctypes.data_as(_abi.f64p), vp, C.byref(rep)),
                    "bsg_batch_lanczos")
        report = {k: getattr(rep, k) for k, _ in rep._fields_}
        return ev.reshape(len(self.tables), nkeep), ([v.T.copy() for v in vecs] if vecs else None), report
