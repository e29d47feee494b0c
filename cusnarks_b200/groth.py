"""Groth16 proving on the GPU: resident proving keys, proofs, and synthetic circuits.

``Prover`` wraps the C ABI (cs_pk_create / cs_prove): the proving key is uploaded once and
stays in HBM; each proof takes a witness (host or device) and the blinding scalars r, s.

``SyntheticCircuit`` builds the benchmark circuit of the configurations quoted for this
path (no public circuit is involved): nConstraints = m - (nPublic + 1) so the QAP domain is
exactly m = 2^k; wire 0 is the constant one, wires 1..nPublic are public inputs, then
private random inputs, then one output wire per constraint.  Each constraint has an A row
and a B row of 3 nonzeros with uniform random Fr coefficients at random wires that are
already defined (earlier inputs or outputs, drawn uniformly from all wires below the
constraint's layer), and its C row selects its output wire, whose value is set to
(A.w)(B.w) so the witness satisfies every constraint.  Outputs are computed layer by layer
on the GPU.  ``setup_pk`` derives a proving key from seeded toxic waste exactly as Groth16
setup defines it (the reference's groth_setup.py), with the field and curve work on the GPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import lib, check, PkDesc, CsError, CS_ERR_NOMEM
from .context import Context
from . import synth

R = synth.R
Q = synth.Q
MONT = 1 << 256


def _t(a):
    """Host array -> device tensor, complete before the library's own streams read it."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()
    torch.cuda.current_stream().synchronize()
    return t


def _np(t):
    return t.cpu().numpy().view(np.uint32)


def _vp(x):
    return ctypes.c_void_p(x)


# ------------------------------------------------------------------- mpoly layout ----
def mpoly_from_entries(n_wires: int, wire: np.ndarray, cons: np.ndarray, coeff: np.ndarray) -> np.ndarray:
    """The reference's by-wire QAP matrix layout (src/cuda/mpoly.cpp:195):
    [n_wires][count per wire][per wire: constraint indices, then 8-word coefficients]."""
    order = np.argsort(wire, kind="stable")
    wire = wire[order]
    cons = cons[order].astype(np.uint32)
    coeff = np.ascontiguousarray(coeff[order], dtype=np.uint32).reshape(-1, 8)
    counts = np.bincount(wire, minlength=n_wires).astype(np.int64)
    start = np.concatenate([[0], np.cumsum(counts)[:-1]])
    E = int(counts.sum())
    out = np.zeros(1 + n_wires + 9 * E, dtype=np.uint32)
    out[0] = n_wires
    out[1:1 + n_wires] = counts
    base = 1 + n_wires + 9 * start                       # per wire block start
    rank = np.arange(E) - start[wire]                    # rank within its wire
    out[base[wire] + rank] = cons
    vpos = base[wire] + counts[wire] + 8 * rank
    idx = vpos[:, None] + np.arange(8)[None, :]
    out[idx.reshape(-1)] = coeff.reshape(-1)
    return out


class CircuitPlan:
    """The host-side draws of the benchmark circuit (no device work): sizes, layers, the
    A and B rows' wires, their coefficients (normal form) and the random inputs, drawn from
    one seeded PCG64 stream in a fixed order, so every builder of the circuit from the
    same seed gets the same circuit."""

    def __init__(self, log_m: int, seed: int = 1, n_public: int = 1, n_inputs: int = 64):
        self.log_m = log_m
        self.m = m = 1 << log_m
        self.n_public = n_public
        self.n_constraints = nc = m - n_public - 1
        n_inputs = max(n_inputs, n_public + 2)
        self.n_inputs = n_inputs
        self.n_vars = n_inputs + nc
        rng = np.random.Generator(np.random.PCG64(seed))
        # Layers of S constraints; a constraint reads wires below the first output of its
        # layer, so the witness is computed layer by layer.  One A index and one B index
        # of each constraint are forced onto the previous layer's wires (a bijection when
        # the layers have equal size), so every wire except the last layer's outputs
        # (S of them) appears in A and in B, as in a real circuit; the other two indices
        # are uniform over the available wires.
        S = 1 << max(6, (log_m + 4) // 2)
        bounds = []
        c0, prev0, prev_n = 0, 0, n_inputs
        while c0 < nc:
            c1 = min(nc, c0 + S)
            bounds.append((c0, c1, n_inputs + c0, prev0, prev_n))
            prev0, prev_n = n_inputs + c0, c1 - c0
            c0 = c1
        self.layers = bounds
        hi = np.empty(nc, dtype=np.int64)
        fa = np.empty(nc, dtype=np.int64)
        fb = np.empty(nc, dtype=np.int64)
        for c0, c1, av, p0, pn in bounds:
            j = np.arange(c1 - c0)
            hi[c0:c1] = av
            fa[c0:c1] = p0 + j % pn
            fb[c0:c1] = p0 + (7 * j + 3) % pn
        self.a_wire = rng.integers(0, hi[:, None], size=(nc, 3)).astype(np.uint32)
        self.b_wire = rng.integers(0, hi[:, None], size=(nc, 3)).astype(np.uint32)
        self.a_wire[:, 0] = fa
        self.b_wire[:, 1] = fb
        # coefficients uniform in Fr (normal form; the matrices hold them in Montgomery form)
        self.coeff = synth.random_field(rng, 6 * nc)
        self.inputs = synth.random_field(rng, n_inputs - 1)

    def initial_witness(self) -> np.ndarray:
        """(n_vars, 8): the constant one, the random inputs, zeros for the outputs."""
        w = np.zeros((self.n_vars, 8), dtype=np.uint32)
        w[0, 0] = 1
        w[1:self.n_inputs] = self.inputs
        return w

    def matrices(self, a_coeff_m: np.ndarray, b_coeff_m: np.ndarray):
        """polsA, polsB, polsC in the reference's by-wire layout from the Montgomery-form
        coefficients (nc, 3, 8); A gets the public-input rows (extend)."""
        nc, nv, npub = self.n_constraints, self.n_vars, self.n_public
        one_m = synth.to_limbs(MONT % R)
        cons = np.repeat(np.arange(nc, dtype=np.uint32), 3)
        ext_w = np.arange(npub + 1, dtype=np.uint32)
        polsA = mpoly_from_entries(
            nv, np.concatenate([self.a_wire.reshape(-1), ext_w]),
            np.concatenate([cons, nc + ext_w]),
            np.concatenate([a_coeff_m.reshape(-1, 8), np.tile(one_m, (npub + 1, 1))]))
        polsB = mpoly_from_entries(nv, self.b_wire.reshape(-1), cons, b_coeff_m.reshape(-1, 8))
        out_w = (self.n_inputs + np.arange(nc)).astype(np.uint32)
        polsC = mpoly_from_entries(nv, out_w, np.arange(nc, dtype=np.uint32), np.tile(one_m, (nc, 1)))
        return polsA, polsB, polsC


class SyntheticCircuit:
    def __init__(self, ctx: Context, log_m: int, seed: int = 1, n_public: int = 1, n_inputs: int = 64):
        plan = CircuitPlan(log_m, seed, n_public, n_inputs)
        self.ctx = ctx
        for k in ("log_m", "m", "n_public", "n_constraints", "n_inputs", "n_vars", "layers", "a_wire", "b_wire"):
            setattr(self, k, getattr(plan, k))
        nc, n_inputs = self.n_constraints, self.n_inputs
        L = lib()
        # coefficients to Montgomery form on the GPU
        d = _t(plan.coeff)
        ctx.field_op_device("to_mont", 1, d.data_ptr(), 0, d.data_ptr(), 6 * nc)
        ctx.sync()
        coeff_m = _np(d).reshape(nc, 6, 8)
        self.a_coeff = np.ascontiguousarray(coeff_m[:, :3])
        self.b_coeff = np.ascontiguousarray(coeff_m[:, 3:])
        # witness: constant one, random inputs, then outputs layer by layer on the GPU
        dw = _t(plan.initial_witness())
        da_wire, db_wire = _t(self.a_wire.reshape(-1)), _t(self.b_wire.reshape(-1))
        da_coeff, db_coeff = _t(self.a_coeff.reshape(-1)), _t(self.b_coeff.reshape(-1))
        doff = _t(np.arange(0, 3 * nc + 1, 3, dtype=np.uint32))
        for c0, c1, *_ in plan.layers:
            check(L.cs_r1cs_layer_eval(ctx.handle, _vp(doff.data_ptr() + 4 * c0), _vp(da_wire.data_ptr()),
                                       _vp(da_coeff.data_ptr()), _vp(doff.data_ptr() + 4 * c0),
                                       _vp(db_wire.data_ptr()), _vp(db_coeff.data_ptr()), c1 - c0,
                                       _vp(dw.data_ptr()), _vp(dw.data_ptr() + 32 * (n_inputs + c0))),
                  ctx.handle)
        ctx.sync()
        self.w = _np(dw).reshape(self.n_vars, 8).copy()
        self.d_w = dw
        self.polsA, self.polsB, self.polsC = plan.matrices(self.a_coeff, self.b_coeff)

    @property
    def public_inputs(self) -> np.ndarray:
        return self.w[1:self.n_public + 1]


def _inv(x: int) -> int:
    return pow(x, -1, R)


def toxic_waste(seed: int):
    """(t, alpha, beta, gamma, delta), uniform in Fr from a seeded PCG64 stream."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return tuple(synth.from_limbs(x) for x in synth.random_field(rng, 5))


def setup_pk(ctx: Context, circ: SyntheticCircuit, seed: int = 7) -> dict:
    """Proving and verifying key from seeded toxic waste (t, alpha, beta, gamma, delta)."""
    import torch
    L = lib()
    # the library's kernels run asynchronously on the context stream: every temporary
    # they read stays referenced here until the final synchronisation
    keep = []
    t, alpha, beta, gamma, delta = toxic_waste(seed)
    m, nv, npub = circ.m, circ.n_vars, circ.n_public
    mont = lambda x: synth.to_limbs((x * MONT) % R)  # noqa: E731
    dt = _t(mont(t))
    dL = torch.empty((m, 8), dtype=torch.int32, device="cuda")
    check(L.cs_setup_lagrange(ctx.handle, circ.log_m, _vp(dt.data_ptr()), _vp(dL.data_ptr())), ctx.handle)
    uvw = []
    for pol in (circ.polsA, circ.polsB, circ.polsC):
        dp = _t(pol)
        keep.append(dp)
        out = torch.empty((nv, 8), dtype=torch.int32, device="cuda")
        check(L.cs_setup_wire_eval(ctx.handle, _vp(dp.data_ptr()), nv, _vp(dL.data_ptr()), m, _vp(out.data_ptr())),
              ctx.handle)
        uvw.append(out)
    ctx.sync()
    du, dv, dw = uvw
    # normal-form copies of u, v for the fixed-base multiplications
    nu = torch.empty_like(du); nvv = torch.empty_like(dv)
    keep += [du, dv, dw, nu, nvv]
    ctx.field_op_device("from_mont", 1, du.data_ptr(), 0, nu.data_ptr(), nv)
    ctx.field_op_device("from_mont", 1, dv.data_ptr(), 0, nvv.data_ptr(), nv)
    g1 = _t(synth.g1_generator())
    g2 = _t(synth.g2_generator())

    def fixed(scal, n, ec2=False):
        keep.append(scal)
        out = torch.empty((n, 32 if ec2 else 16), dtype=torch.int32, device="cuda")
        ctx.scmul_device(scal.data_ptr(), (g2 if ec2 else g1).data_ptr(), n, out.data_ptr(), ec2=ec2,
                         point_stride_words=0)
        return out

    def pts_of(vals, ec2=False):
        s = _t(np.stack([synth.to_limbs(v) for v in vals]))
        return fixed(s, len(vals), ec2)

    A = fixed(nu, nv)
    B1 = fixed(nvv, nv)
    B2 = fixed(nvv, nv, ec2=True)
    dal, dbe = _t(mont(alpha)), _t(mont(beta))
    keep += [dt, dL, dal, dbe, g1, g2]
    cs = torch.empty((nv, 8), dtype=torch.int32, device="cuda")
    dk = _t(mont(_inv(delta)))
    keep += [dk, cs]
    check(L.cs_setup_c_scalars(ctx.handle, _vp(du.data_ptr()), _vp(dv.data_ptr()), _vp(dw.data_ptr()),
                               _vp(dal.data_ptr()), _vp(dbe.data_ptr()), _vp(dk.data_ptr()), nv, _vp(cs.data_ptr())),
          ctx.handle)
    C = fixed(cs, nv)
    ics = torch.empty((npub + 1, 8), dtype=torch.int32, device="cuda")
    dkg = _t(mont(_inv(gamma)))
    keep += [dkg, ics]
    check(L.cs_setup_c_scalars(ctx.handle, _vp(du.data_ptr()), _vp(dv.data_ptr()), _vp(dw.data_ptr()),
                               _vp(dal.data_ptr()), _vp(dbe.data_ptr()), _vp(dkg.data_ptr()), npub + 1,
                               _vp(ics.data_ptr())), ctx.handle)
    IC = fixed(ics, npub + 1)
    zt = (pow(t, m, R) - 1) % R
    dkh = _t(mont(zt * _inv(delta) % R))
    hs = torch.empty((m - 1, 8), dtype=torch.int32, device="cuda")
    keep += [dkh, hs]
    check(L.cs_setup_pow_scalars(ctx.handle, _vp(dt.data_ptr()), _vp(dkh.data_ptr()), m - 1, _vp(hs.data_ptr())),
          ctx.handle)
    H = fixed(hs, m - 1)
    alpha1, beta1, delta1 = (pts_of([v]) for v in (alpha, beta, delta))
    beta2, gamma2, delta2 = (pts_of([v], ec2=True) for v in (beta, gamma, delta))
    ctx.sync()
    keep.clear()
    pk = {
        "n_vars": nv, "n_public": npub, "domain_size": m,
        "polsA": circ.polsA, "polsB": circ.polsB,
        "A": torch.cat([A, alpha1, delta1]), "B1": torch.cat([B1, beta1, delta1]),
        "B2": torch.cat([B2, beta2, delta2]), "C": C, "hExps": H, "delta_1": delta1,
        "vk": {"alpha_1": _np(alpha1).reshape(16), "beta_2": _np(beta2).reshape(32),
               "gamma_2": _np(gamma2).reshape(32), "delta_2": _np(delta2).reshape(32),
               "IC": _np(IC).reshape(-1, 16)},
    }
    return pk


def pk_to_host(pk: dict) -> dict:
    out = {}
    for k, v in pk.items():
        if hasattr(v, "cpu"):
            out[k] = _np(v).reshape(v.shape[0], -1)
        else:
            out[k] = v
    return out


class Prover:
    """A proving key resident in HBM and the prove call (cs_pk_create / cs_prove)."""

    def __init__(self, ctx: Context, pk: dict, fixed_base: int = 0):
        """fixed_base: window of the resident fixed-base MSM tables (0 = automatic per MSM,
        negative = no tables: every proof runs the generic MSM over the key's points)."""
        import torch
        self.ctx = ctx
        self._keep = []
        on_device = hasattr(pk["A"], "data_ptr")

        def ptr(a):
            if hasattr(a, "data_ptr"):
                return a.data_ptr()
            arr = np.ascontiguousarray(a, dtype=np.uint32)
            self._keep.append(arr)
            return arr.ctypes.data

        pa, pb = pk["polsA"], pk["polsB"]
        if on_device:
            pa_t, pb_t = _t(pa), _t(pb)
            self._keep += [pa_t, pb_t]
            pa_p, pb_p = pa_t.data_ptr(), pb_t.data_ptr()
        else:
            pa_p, pb_p = ptr(pa), ptr(pb)
        ent = lambda p: int(np.asarray(p[1:1 + int(p[0])], dtype=np.int64).sum())  # noqa: E731
        d = PkDesc(pk["n_vars"], pk["n_public"], pk["domain_size"],
                   pa_p, len(pa), ent(pa), pb_p, len(pb), ent(pb),
                   ptr(pk["A"]), ptr(pk["B1"]), ptr(pk["B2"]), ptr(pk["C"]), ptr(pk["hExps"]), ptr(pk["delta_1"]))
        h = ctypes.c_void_p()
        check(lib().cs_pk_create(ctx.handle, ctypes.byref(d), 1 if on_device else 0, ctypes.byref(h)), ctx.handle)
        self.handle = h
        self.n_vars = pk["n_vars"]
        self._keep.clear()
        del torch
        self.fixed_base_note = None
        if fixed_base >= 0:
            try:
                self.set_fixed_base(fixed_base)
            except CsError as e:
                # automatic tables (~13x the key's points) that do not fit in device memory:
                # the key stays without them and proofs run the generic MSM over its points
                if fixed_base != 0 or e.code != CS_ERR_NOMEM:
                    raise
                self.fixed_base_note = f"fixed-base tables left out: {e}"

    def set_fixed_base(self, window: int = 0):
        """Builds (window >= 0) or drops (window < 0) the key's fixed-base tables."""
        check(lib().cs_pk_fixed_base(self.ctx.handle, self.handle, window), self.ctx.handle)

    def fixed_windows(self) -> list:
        """Windows of the A, B1, B2, C, H tables (0 = no table)."""
        return [int(lib().cs_pk_fixed_window(self.handle, k)) for k in range(5)]

    def stages(self) -> dict:
        """Stage completion times (ms) of the last finished proof on this prover's context."""
        out = (ctypes.c_float * 7)()
        check(lib().cs_ctx_prove_stages(self.ctx.handle, out, 7), self.ctx.handle)
        keys = ("A", "B1", "B2", "C", "hstep", "H", "total")
        return {k: round(float(v), 3) for k, v in zip(keys, out)}

    def device_bytes(self) -> int:
        return int(lib().cs_pk_device_bytes(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            lib().cs_pk_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def prove(self, w, r, s) -> np.ndarray:
        """w: (n_vars, 8) normal form; r, s: 8-word normal form.  Returns 64 words:
        pi_A (16) | pi_B (32) | pi_C (16), affine Montgomery."""
        w = np.ascontiguousarray(w, dtype=np.uint32).reshape(-1, 8)
        assert w.shape[0] == self.n_vars
        r = np.ascontiguousarray(r, dtype=np.uint32).reshape(8)
        s = np.ascontiguousarray(s, dtype=np.uint32).reshape(8)
        out = np.zeros(64, dtype=np.uint32)
        check(lib().cs_prove(self.ctx.handle, self.handle, w.ctypes.data, r.ctypes.data, s.ctypes.data,
                             out.ctypes.data), self.ctx.handle)
        return out

    def prove_batch_device(self, d_ws, rs, ss, d_proofs):
        """Several proofs in one pass (cs_prove_batch_device): d_ws, d_proofs device pointers,
        rs, ss 8-word normal-form scalars, one per proof."""
        k = len(d_ws)
        w_arr = (ctypes.c_void_p * k)(*d_ws)
        p_arr = (ctypes.c_void_p * k)(*d_proofs)
        r = np.ascontiguousarray(np.stack([np.asarray(x, dtype=np.uint32).reshape(8) for x in rs]))
        s = np.ascontiguousarray(np.stack([np.asarray(x, dtype=np.uint32).reshape(8) for x in ss]))
        check(lib().cs_prove_batch_device(self.ctx.handle, self.handle, k, ctypes.cast(w_arr, ctypes.c_void_p),
                                          r.ctypes.data, s.ctypes.data, ctypes.cast(p_arr, ctypes.c_void_p)),
              self.ctx.handle)

    def prove_device(self, d_w: int, r, s, d_proof: int):
        r = np.ascontiguousarray(r, dtype=np.uint32).reshape(8)
        s = np.ascontiguousarray(s, dtype=np.uint32).reshape(8)
        check(lib().cs_prove_device(self.ctx.handle, self.handle, _vp(d_w), r.ctypes.data, s.ctypes.data,
                                    _vp(d_proof)), self.ctx.handle)
