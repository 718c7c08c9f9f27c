"""Learned W_c(q, i w) frequency interpolator with validation and fallback.

There is no counterpart in the reference: it computes chi0 and W at every
point of the imaginary-frequency grid (x0kf per frequency, then
m_llw.f90:265-376).  Here the plain method computes W_c exactly at the
frequency w = 0, at a few anchor frequencies and at a few held-out
frequencies; a network predicts W_c at the other grid points:

  * full matrix: a per-target linear head (bank 1) on the normalised anchor
    values of every element;
  * dominant block (the top nb eigenvectors of v, where W_c is largest):
    a second per-target head (bank 0) plus an MLP correction
    (16-256-256-1, BF16 weights).
Element features of the dominant block: log10 of the Coulomb eigenvalue of
the element's row and column (/3), re/im, diagonal.  Both heads start from linear interpolation in
the Gauss-Legendre coordinate x, are then set by weighted least squares, and
bank 0 and the MLP are trained with Adam.

Training data: exact W_c of other q points on the whole grid: their
dominant block (bank 0) and a fixed block of random rows x random columns
(bank 1).  Every step (projection, features, normal equations, forward,
backward, Adam, head, scatter) runs in this library's own kernels.

Validation: the network also predicts the held-out frequencies; the
imaginary-axis Sigma_c change that the prediction error there causes,
scaled by n_pred / n_held, estimates the QP-energy error (largest over
the states).  Above the tolerance (1 meV) the q point falls back to the plain
method at every frequency.

W_c slots on the device: (nslot, N, N) complex, slot 0 = w = 0, slot 1 + i =
grid point i (the reference's __WVR first record and __WVI records).
"""
import math
import time

import numpy as np

from . import lib, synth

HARTREE_EV = 27.211386245988


def split_grid(nw=48, anchors=(0, 6, 13, 20, 27, 34, 41, 47), nheld=8):
    """Anchor, target (predicted) and held-out grid indices (0-based)."""
    anchors = tuple(int(a) for a in anchors)
    targets = [i for i in range(nw) if i not in anchors]
    held = targets[2::5][:nheld]
    return list(anchors), targets, held


def lib_offsets():
    """Parameter layout of the library's network (16 inputs, 256 hidden, 128 head rows)."""
    nin, nh, ntmax = 16, 256, 128
    off_c = nin * nh + nh + nh * nh + nh + nh + 1
    assert off_c + ntmax * nin == lib.wsurr_nparam()
    return dict(NIN=nin, NH=nh, NTMAX=ntmax, NMLP=64, OFF_C=off_c, OFF_W3=off_c - 1 - nh, OFF_B3=off_c - 1)


def linear_head_init(x, anchors, targets, p, banks=(0, 64)):
    """Head rows (one per target in each bank) = linear interpolation in x
    between the neighbouring anchors."""
    o = lib_offsets()
    nin = o["NIN"]
    xa = np.asarray(x)[anchors]
    for j, t in enumerate(targets):
        i = int(np.clip(np.searchsorted(xa, x[t]) - 1, 0, len(anchors) - 2))
        a = (x[t] - xa[i]) / (xa[i + 1] - xa[i])
        row = np.zeros(nin, np.float32)
        row[i], row[i + 1] = 1.0 - a, a
        for b0 in banks:
            p[o["OFF_C"] + (b0 + j) * nin: o["OFF_C"] + (b0 + j + 1) * nin] = row
    return p


def without_mlp(p):
    """The same parameters with the MLP output switched off (W3 = 0, b3 = 0)."""
    o = lib_offsets()
    q = p.copy()
    q[o["OFF_W3"]:o["OFF_C"]] = 0.0
    return q


class Workload:
    """Exact W_c generator of the Sigma_c configuration (chi0 of the Lorentzian
    model, then W = (1 - v chi0)^-1 v - v in the Coulomb eigenbasis)."""

    def __init__(self, N=600, nk=64, nocc=4, nun=(40, 60), nw=48, seed=20263, torch=None):
        import torch as _torch
        self.torch = torch or _torch
        self.N, self.nk, self.nocc, self.nun, self.nw, self.seed = N, nk, nocc, nun, nw, seed
        mesh = synth.imag_mesh(nw)
        self.mesh = mesh
        self.freq = np.concatenate([[0.0], mesh["freq_i"]])          # slot frequencies
        self.xslot = np.concatenate([[1.0], mesh["x"]]).astype(np.float32)
        vsq, q = synth.coulomb(N, seed + 1)
        self.vsq = vsq
        self.m2e = lib.to_device(q)
        self.idx_order = np.argsort(-vsq)                            # dominant eigenvectors first

    def q_inputs(self, iq):
        rng = np.random.default_rng(self.seed * 1000 + iq)
        nocc_a, nun_a, eocc, eun = synth.chi0_spectrum(rng, self.nk, self.nocc, self.nun)
        npair = int(np.sum(nocc_a * nun_a))
        g = self.torch.Generator(device="cuda")
        g.manual_seed(self.seed * 7919 + iq)
        z = self.torch.randn(2 * self.N * npair, dtype=self.torch.float64, device="cuda", generator=g)
        z = self.torch.view_as_complex((z / math.sqrt(self.N)).view(-1, 2)).contiguous()
        return dict(nocc=nocc_a, nun=nun_a, eocc=np.concatenate(eocc) * 0.5, eun=np.concatenate(eun) * 0.5, z=z,
                    npair=npair)

    def exact(self, iq, slots, out=None, inp=None):
        """Exact W_c of q point iq at the given slots -> (len(slots), N, N) complex128 device tensor,
        or written into out[slots] when out (nslot, N, N) is given."""
        t, N = self.torch, self.N
        inp = inp or self.q_inputs(iq)
        slots = list(slots)
        ns = len(slots)
        chi = t.zeros(N * N * ns, dtype=t.complex128, device="cuda")
        lib.chi0_lorentz_d(chi, N, ns, self.freq[slots], self.nk, inp["nocc"], inp["nun"], inp["eocc"], inp["eun"],
                           inp["z"])
        w = t.zeros(N * N * ns, dtype=t.complex128, device="cuda")
        lib.wvi_llw(chi, 2, self.vsq, self.m2e, True, False, 2, zw=w, device=True, ngb=N, niw=ns)
        del chi
        w = w.view(ns, N, N)
        if out is None:
            return w
        if slots == list(range(slots[0], slots[0] + ns)):
            out[slots[0]:slots[0] + ns] = w
        else:
            out[t.tensor(slots, device="cuda")] = w
        return out


class WcSurrogate:
    """The network and the data it is trained on (one per process: the
    library holds one set of parameters).

    Head bank 0 (rows 0..63, with the MLP term) serves the dominant block
    (the top nb eigenvectors of v); bank 1 (rows 64..127, linear only) serves
    the whole matrix.  Training samples: the dominant block of each training
    q point, and a block of random rows x random columns for bank 1."""

    FULL = 64

    def __init__(self, work, anchors, targets, nb=64, seed=1234):
        t = work.torch
        self.work, self.t = work, t
        self.anchors, self.targets = list(anchors), list(targets)
        if len(self.targets) > 64 or len(self.anchors) > 14:
            raise ValueError("at most 64 targets and 14 anchors")
        self.aslot = [1 + a for a in self.anchors]
        self.nb = nb
        self.idx = np.sort(work.idx_order[:nb]).astype(np.int32)
        self.ne = 2 * nb * nb
        self.rng = np.random.default_rng(seed)
        # element feature per Coulomb eigen-index: log10 of the eigenvalue of v, / 3
        self.ftab = (np.log10(np.asarray(work.vsq) ** 2) / 3.0).astype(np.float32)
        # rows and columns of the training block of the full-matrix bank
        self.rand_r = np.sort(self.rng.choice(work.N, nb, replace=False)).astype(np.int32)
        self.rand_c = np.sort(self.rng.choice(work.N, nb, replace=False)).astype(np.int32)
        lib.wsurr_init(seed)
        p = linear_head_init(work.mesh["x"], self.anchors, self.targets, lib.wsurr_params())
        lib.wsurr_params(p)
        self.p_linear = p.copy()
        self.proj = {0: [], self.FULL: []}

    # ---- data
    def _project(self, w_slots, ridx, cidx=None):
        t = self.t
        ns = w_slots.shape[0]
        pr = t.empty(ns * self.ne, dtype=t.float32, device="cuda")
        lib.wsurr_project_d(w_slots, self.work.N, ns, ridx, pr, cidx)
        return pr.view(1, ns, self.ne)

    def add_training_q(self, w_slots):
        """Project the exact W_c (nslot, N, N) of one q point: its dominant
        block and the block of random rows x random columns."""
        self.proj[0].append(self._project(w_slots, self.idx))
        self.proj[self.FULL].append(self._project(w_slots, self.rand_r, self.rand_c))

    def samples(self, proj, bank=0, targets=None, with_y=True):
        t = self.t
        targets = self.targets if targets is None else list(targets)
        tsl = [1 + i for i in targets]
        thead = [bank + self.targets.index(i) for i in targets]
        nq, ns, ne = proj.shape
        n = nq * ne * len(tsl)
        d = dict(n=n, nt=len(tsl), thead=thead, x=t.empty(n * 16, dtype=t.float32, device="cuda"),
                 tix=t.empty(n, dtype=t.int32, device="cuda"),
                 scale=t.empty(n, dtype=t.float32, device="cuda"))
        if with_y:
            d["y"] = t.empty(n, dtype=t.float32, device="cuda")
            d["w"] = t.empty(n, dtype=t.float32, device="cuda")
        # element features on the dominant block only (they do not help the linear full-matrix bank)
        ftab = self.ftab if bank == 0 else None
        lib.wsurr_features_d(proj, nq, ns, ne, self.aslot, tsl, thead, self.work.xslot, d["x"], d["tix"],
                             d.get("y"), d.get("w"), d["scale"], rid=self.idx, cid=self.idx, ftab=ftab)
        return d

    # ---- training
    def train(self, schedule=((1e-3, 2000), (3e-4, 1500), (1e-4, 1000)), batch=8192, seed=7, ridge=1e-9):
        """Least squares of both head banks, then Adam on the dominant-block
        bank (head rows and MLP); the full-matrix bank keeps its least-squares rows."""
        t = self.t
        t0 = time.time()
        for b in (self.FULL, 0):
            d = self.samples(t.cat(self.proj[b]), bank=b)
            lib.wsurr_lsq_accumulate_d(d["x"], d["y"], d["w"], d["n"], d["thead"])
        self.rows_lsq = lib.wsurr_lsq_solve(ridge)
        self.p_lsq = without_mlp(lib.wsurr_params())
        n = d["n"]
        log = []
        for k, (lr, steps) in enumerate(schedule):
            loss = lib.wsurr_train_d(d["x"], d["tix"], d["y"], d["w"], n, batch, steps, lr, seed + k)
            log.append((lr, steps, loss))
        lib.synchronize()
        self.train_seconds = time.time() - t0
        self.train_samples = n
        return log

    # ---- inference
    def predict(self, w_slots, targets=None):
        """Fill the target slots of w_slots (nslot, N, N) from its anchor slots:
        bank 1 (linear) on the whole matrix, then bank 0 + MLP on the dominant block."""
        t = self.t
        targets = self.targets if targets is None else list(targets)
        tsl = [1 + i for i in targets]
        N, ns = self.work.N, w_slots.shape[0]
        thead = [self.FULL + self.targets.index(i) for i in targets]
        lib.wsurr_head_full_d(w_slots, N, N, ns, self.aslot, tsl, thead, self.work.xslot[tsl])
        d = self.samples(self._project(w_slots, self.idx), 0, targets, with_y=False)
        out = t.empty(d["n"], dtype=t.float32, device="cuda")
        lib.wsurr_forward_d(d["x"], d["tix"], out, d["n"])
        lib.wsurr_scatter_d(w_slots, N, ns, self.idx, tsl, out, d["scale"])
        return w_slots


class SigmaProbe:
    """Imaginary-axis Sigma_c of one q point's task (40 target x 400
    intermediate states, Sigma_c configuration generator) for W_c slot stacks,
    through this library's correlation block with the real-axis W set to zero.
    The imaginary-axis weights of a grid point depend on that point alone
    (m_sxcf_gemm.f90:446-451), so a sub-grid gives that sub-grid's share; the
    w = 0 slot only enters the sum through the point 0 weight, which is not
    used for differences (their w = 0 slot is exact, hence zero)."""

    def __init__(self, work, iq, ntq=40, nm=400, nreal=50):
        from . import sched
        t, N = work.torch, work.N
        self.work, self.t = work, t
        rng = np.random.default_rng(work.seed * 31 + iq)
        self.omega = np.sort(rng.uniform(-1.0, 1.0, ntq))
        self.ekc = np.sort(rng.uniform(-1.0, 4.0, nm))
        g = t.Generator(device="cuda")
        g.manual_seed(work.seed * 104729 + iq)
        z = t.randn(2 * N * nm * ntq, dtype=t.float64, device="cuda", generator=g) / math.sqrt(N)
        self.zmel = t.view_as_complex(z.view(-1, 2)).contiguous()
        self.fr = synth.freq_r_mesh(nreal)
        self.ef, self.esmr = 0.0, 0.01
        self.nwxi, self.nwx, ntmax = sched.get_nwx(self.omega, self.ekc, self.fr, self.ef, self.esmr)
        self.ns2r = 0                       # no real-axis pole columns: only the imaginary-axis part
        self.wr = t.zeros(N * N * nreal, dtype=t.complex128, device="cuda")
        self.ntq, self.nm = ntq, nm

    def sigma(self, w_slots, grid):
        """Re diag Sigma_c (Ha) from w_slots (1 + len(grid), N, N): slot 0 = w = 0,
        slot 1 + k = grid point grid[k]."""
        t, m = self.t, self.work.mesh
        grid = list(grid)
        zsec = t.zeros(self.ntq * self.ntq, dtype=t.complex128, device="cuda")
        lib.sxcf_correlation(zsec, self.zmel, 1, self.nm, self.ns2r, self.nwxi, self.nwx, self.ntq,
                             w_slots.reshape(-1), self.wr, self.omega, self.ekc, 0, self.ef, self.esmr, 1.0,
                             m["ua"], m["x"][grid], m["wx"][grid], m["expa"][grid], self.fr,
                             nblochpmx=self.work.N, device=True, ngb=self.work.N, ntq=self.ntq)
        return t.real(zsec.view(self.ntq, self.ntq).diagonal()).cpu().numpy()

    def delta(self, dw_slots, grid):
        """Sigma_c change from W_c differences on the grid points only (slot 0 ignored)."""
        t = self.t
        N = self.work.N
        buf = t.zeros((1 + len(grid), N, N), dtype=t.complex128, device="cuda")
        buf[1:] = dw_slots
        return self.sigma(buf, grid)


def qp_mev(dsig, sig_ref, scale_ev=5.0):
    """QP-energy error (meV) with Sigma_c normalised to a mean |Re Sigma_c,nn| of scale_ev."""
    return float(np.max(np.abs(dsig)) / np.mean(np.abs(sig_ref)) * scale_ev * 1e3)


def _ms(t, fn):
    """Run fn on the current stream between CUDA events; returns (result, ms)."""
    e0, e1 = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
    t.cuda.synchronize()
    e0.record()
    r = fn()
    e1.record()
    t.cuda.synchronize()
    return r, e0.elapsed_time(e1)


def surrogate_w(sur, work, probe, iq, held, tol_mev=1.0, sig_scale=None, inp=None):
    """W_c of q point iq on the whole grid by the surrogate path: exact at w = 0,
    the anchors and the held-out points, predicted elsewhere; validated on the
    held-out points, recomputed exactly at every predicted point when the
    estimated QP error exceeds tol_mev.  Returns (w_slots, report); the report
    holds the device time of each phase (ms)."""
    t, N, nw = work.torch, work.N, work.nw
    inp = inp or work.q_inputs(iq)
    pred = [i for i in sur.targets if i not in held]
    exact_slots = [0] + sur.aslot + [1 + h for h in held]
    ev = [t.cuda.Event(enable_timing=True) for _ in range(5)]
    ev[0].record()
    w = t.zeros((nw + 1, N, N), dtype=t.complex128, device="cuda")
    work.exact(iq, exact_slots, out=w, inp=inp)
    ev[1].record()
    hs = t.tensor([1 + h for h in held], device="cuda")
    wheld = w[hs].clone()
    sur.predict(w)
    ev[2].record()
    dsig_held = probe.delta(w[hs] - wheld, held)
    w[hs] = wheld
    ev[3].record()
    if sig_scale is None:
        sig_scale = probe.sigma(w, range(nw))
    # the held-out points sample the predicted ones (midway between anchors,
    # where interpolation errors peak): their Sigma_c change, scaled by
    # n_pred / n_held, estimates the change from all predicted points
    est = qp_mev(dsig_held, sig_scale) * len(pred) / len(held)
    fallback = est > tol_mev
    if fallback:
        work.exact(iq, [1 + i for i in pred], out=w, inp=inp)
    ev[4].record()
    t.cuda.synchronize()
    phases = dict(exact_ms=ev[0].elapsed_time(ev[1]), predict_ms=ev[1].elapsed_time(ev[2]),
                  validate_ms=ev[2].elapsed_time(ev[3]), fallback_ms=ev[3].elapsed_time(ev[4]))
    return w, dict(est_mev=est, fallback=bool(fallback), n_exact=len(exact_slots) + (len(pred) if fallback else 0),
                   **phases)


def prediction_errors(sur, work, probe, wex, sig, pred, params):
    """Errors of the network with the given parameters at the predicted grid
    points, W_c predicted from the exact anchors: full-matrix and
    dominant-block relative Frobenius errors and the QP error (meV)."""
    t = work.torch
    lib.wsurr_params(params)
    ps = t.tensor([1 + i for i in pred], device="cuda")
    blk = t.tensor(sur.idx.astype(np.int64), device="cuda")
    w = wex.clone()
    w[ps] = 0
    sur.predict(w, targets=pred)
    dw = (w - wex)[ps]
    ref = wex[ps]
    r = dict(w_rel=float(t.linalg.vector_norm(dw) / t.linalg.vector_norm(ref)),
             w_rel_block=float(t.linalg.vector_norm(dw[:, blk][:, :, blk])
                               / t.linalg.vector_norm(ref[:, blk][:, :, blk])),
             qp_mev=qp_mev(probe.delta(dw, pred), sig))
    del w, dw
    return r


def study(N=600, nq_train=48, nq_test=16, nw=48, nb=64, schedule=((1e-3, 2000), (3e-4, 1500), (1e-4, 1000)),
          tol_mev=1.0, seed=20263, nm=400, ntq=40, precision="split", log=None, nslices=3):
    """Train on exact W_c of nq_train q points, then run the surrogate path on
    nq_test other q points and compare with the plain method (all frequencies
    exact).  Per test q: errors of the linear interpolation the heads start
    from, of the least-squares heads alone, and of the trained network; the
    surrogate path's validation estimate, fallback and time against the
    plain method's (in FP64 and in the path's precision)."""
    import torch as t
    log = log or (lambda m: None)
    if t.cuda.current_stream().cuda_stream == 0:
        lib.share_torch_stream()
    # "split" / "split-f16": FP16 slices; "split-i8": nslices int8 slices (Ozaki); "fp64": plain
    prec = {"split": (lib.PREC_SPLIT_F16, 2), "split-f16": (lib.PREC_SPLIT_F16, 2),
            "split-i8": (lib.PREC_SPLIT_I8, nslices), "fp64": (lib.PREC_FP64, 1)}[precision]
    lib.set_precision(*prec)
    work = Workload(N=N, nw=nw, seed=seed)
    anchors, targets, held = split_grid(nw)
    pred = [i for i in targets if i not in held]
    sur = WcSurrogate(work, anchors, targets, nb=nb)
    allslots = list(range(nw + 1))
    t0 = time.time()
    for iq in range(nq_train):
        sur.add_training_q(work.exact(iq, allslots))
    t.cuda.synchronize()
    log(f"training data: {nq_train} q x {nw + 1} slots in {time.time() - t0:.1f}s")
    tr_log = sur.train(schedule)
    log(f"training: {sur.train_samples} samples, least squares on {sur.rows_lsq} head rows, "
        f"{sum(s for _, s in schedule)} Adam steps, {sur.train_seconds:.1f}s, last loss {tr_log[-1][2]:.3e}")
    p_trained = lib.wsurr_params()
    variants = dict(linear=without_mlp(sur.p_linear), lsq=sur.p_lsq, trained=p_trained)
    rows = []
    ps = t.tensor([1 + i for i in pred], device="cuda")
    for iq in range(nq_train, nq_train + nq_test):
        inp = work.q_inputs(iq)
        probe = SigmaProbe(work, iq, ntq=ntq, nm=nm)
        lib.set_precision(lib.PREC_FP64)
        wex64, ms_plain64 = _ms(t, lambda: work.exact(iq, allslots, inp=inp))
        lib.set_precision(*prec)
        wex, ms_plain = _ms(t, lambda: work.exact(iq, allslots, inp=inp))
        sig = probe.sigma(wex, range(nw))
        r = dict(iq=iq, ms_plain=ms_plain, ms_plain_fp64=ms_plain64, sig_mean_abs_ha=float(np.mean(np.abs(sig))))
        for name, prm in variants.items():
            r[name] = prediction_errors(sur, work, probe, wex, sig, pred, prm)
        lib.wsurr_params(p_trained)
        (wsur, rep), ms_sur = _ms(t, lambda: surrogate_w(sur, work, probe, iq, held, tol_mev, sig, inp))
        r.update(rep, ms_surrogate=ms_sur)
        r["qp_mev_final"] = qp_mev(probe.delta((wsur - wex)[ps], pred), sig)
        lib.set_precision(lib.PREC_FP64)
        sig64 = probe.sigma(wex64, range(nw))
        lib.set_precision(*prec)
        r["qp_mev_final_vs_fp64"] = qp_mev(probe.sigma(wsur, range(nw)) - sig64, sig64)
        rows.append(r)
        log(f"q {iq}: W rel linear {r['linear']['w_rel']:.2e} lsq {r['lsq']['w_rel']:.2e} trained "
            f"{r['trained']['w_rel']:.2e} (block {r['linear']['w_rel_block']:.2e} / {r['lsq']['w_rel_block']:.2e} / "
            f"{r['trained']['w_rel_block']:.2e}); QP meV {r['linear']['qp_mev']:.3f} / {r['lsq']['qp_mev']:.3f} / "
            f"{r['trained']['qp_mev']:.3f}; est {r['est_mev']:.3f}, fallback {r['fallback']}, final "
            f"{r['qp_mev_final']:.3f} (vs FP64 plain {r['qp_mev_final_vs_fp64']:.3f}); {ms_sur:.1f} ms "
            f"(exact {r['exact_ms']:.1f}, predict {r['predict_ms']:.1f}, validate {r['validate_ms']:.1f}, "
            f"fallback {r['fallback_ms']:.1f}) vs plain {ms_plain:.1f} ms, plain FP64 {ms_plain64:.1f} ms")
        del wex, wex64, wsur, probe
    lib.set_precision(lib.PREC_FP64)
    return dict(rows=rows, train_log=tr_log, precision=precision, train_seconds=sur.train_seconds, train_samples=sur.train_samples,
                anchors=anchors, held=held, predicted=pred, surrogate=sur, work=work)
