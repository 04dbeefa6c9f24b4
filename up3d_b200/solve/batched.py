"""Many channel cases solved together on one device.

The reference solves one case at a time.  Here the cases' meshes are
concatenated into one mesh of disconnected components, so that every pass
(element sweep, row gather, Term 3, SpMV, AMG V-cycle, Krylov vectors) is
one launch over all cases: small cases no longer leave the GPU idle between
launches.  Each element carries its case index and takes that case's flow
(up3d_residual_jacobian_batched); the Jacobian, the Picard block and the AMG
hierarchy are block diagonal, so the Krylov solution of the joint system is
the per-case solutions.

``solve_newton_batched`` steps all cases in lockstep with the plain driver's
ingredients per case -- Picard seed, exact Jacobian, GMRES(60) + AMG rebuilt
(refreshed) every two steps, Eisenstat-Walker forcing (the smallest over the
active cases), a merit line search with up to five halvings decided per case,
and the Mach continuation as a shared ramp that each case follows up to its
own target.  A case stops moving once its |R_free|_inf is below the
tolerance at its target Mach.  Each case freezes its (upstream, branch)
state once its residual is below ``freeze_tol`` (the plain driver's frozen
finish; the other cases stay live in the same launches) and is accepted on
frozen convergence -- the plain driver's refresh / revert of the frozen state
is not repeated here.

Lockstep pays for small cases, whose solve time is launches and host
synchronisations, and costs for large ones, which fill the GPU alone and
would be tied to the slowest case's iteration count.  ``CaseSet`` therefore
puts the cases below a size into one union and runs the others one by one.
"""

from __future__ import annotations

import ctypes
import time
from typing import Dict, List, Optional, Sequence

import numpy as np

from .. import _lib as L
from ..mesh.kuhn import BumpMesh
from .fused import FlowParams
from .linear import amg_for, solve_cg, solve_gmres, with_dirichlet
from .newton import ChannelWorkspace, _ew_forcing, mach_schedule


class BatchedChannels:
    """The union of several channel meshes on one device.

    ``ordering`` renumbers each case's nodes and elements within its own
    block (``up3d_b200.mesh.order``: "given", "morton", "hilbert"); potentials
    of the union are in that numbering, ``case_phi`` maps a case's block back
    to the case mesh's own numbering.  ``BatchedChannels.tuned`` picks the
    ordering and the launch shapes by timing them."""

    def __init__(self, meshes: Sequence[BumpMesh], u_inf: float = 1.0, ordering: str = "given",
                 tune: bool = True):
        t = L.require_cuda()
        from ..mesh.order import renumber
        self.meshes = list(meshes)
        self.n_cases = len(self.meshes)
        self.ordering = ordering
        self.renum = [renumber(m.nodes, m.elements, ordering) for m in self.meshes]
        node_off = np.cumsum([0] + [m.n_nodes for m in self.meshes])
        elem_off = np.cumsum([0] + [m.n_tets for m in self.meshes])
        nodes = np.concatenate([r.nodes for r in self.renum])
        elements = np.concatenate([r.elements.astype(np.int64) + node_off[c]
                                   for c, r in enumerate(self.renum)]).astype(np.int32)
        dirichlet = np.concatenate([r.node_set(m.dirichlet_nodes) + node_off[c]
                                    for c, (m, r) in enumerate(zip(self.meshes, self.renum))])
        self.node_off, self.elem_off = node_off, elem_off
        self.ws = ChannelWorkspace(nodes, elements, dirichlet, u_inf=u_inf, tune=tune)
        self._node_inv = [t.from_numpy(r.node_inv).cuda() for r in self.renum]
        self._trial = None
        case_e = np.repeat(np.arange(self.n_cases, dtype=np.int32), np.diff(elem_off))
        case_n = np.repeat(np.arange(self.n_cases, dtype=np.int64), np.diff(node_off))
        self.case_of_elem = t.from_numpy(case_e).cuda()
        self.case_of_node = t.from_numpy(case_n).cuda()
        self.n_tets = int(elem_off[-1])
        self.u_inf = float(u_inf)
        self.branch = t.empty(self.n_tets, dtype=t.int8, device="cuda")
        self.up_fz = None   # (E) int64 frozen upstream, once a case freezes
        self.br_fz = None   # (E) int8 frozen branch, -1 = live

    def unfreeze(self, cases):
        """Return the listed cases to the live flux."""
        if self.br_fz is None:
            return
        for c in cases:
            self.br_fz[int(self.elem_off[c]):int(self.elem_off[c + 1])] = -1

    def freeze(self, cases):
        """Freeze the listed cases at the state of the last evaluation."""
        t = L.torch()
        if self.up_fz is None:
            self.up_fz = t.zeros(self.n_tets, dtype=t.int64, device="cuda")
            self.br_fz = t.full((self.n_tets,), -1, dtype=t.int8, device="cuda")
        for c in cases:
            a, b = int(self.elem_off[c]), int(self.elem_off[c + 1])
            self.up_fz[a:b] = self.ws.ev.upstream[a:b].to(t.int64)
            self.br_fz[a:b] = self.branch[a:b]

    def _flows(self, machs):
        arr = (L.Flow * self.n_cases)()
        for c, m in enumerate(machs):
            arr[c] = FlowParams(m_inf=float(m), u_inf=self.u_inf).c()
        return arr

    def evaluate(self, phi, machs, jacobian: bool = True):
        """R (and the Jacobian data, rho~, upstream) of every case at once,
        into the union workspace.  machs=None reuses the Mach numbers of the
        last call (no host synchronisation: capturable for jacobian=False)."""
        ev = self.ws.ev
        L.call("up3d_residual_jacobian_batched", ev.mesh.handle, phi.data_ptr(), self.n_cases,
               None if machs is None else self._flows(machs), self.case_of_elem.data_ptr(),
               L.ptr(self.up_fz), L.ptr(self.br_fz),
               ev.R.data_ptr(), ev.data.data_ptr() if jacobian else None, ev.rho_tilde.data_ptr(),
               ev.upstream.data_ptr(), self.branch.data_ptr(), ev.monitors.data_ptr(), L.stream_ptr())
        return ev.R

    def case_phi(self, phi, c: int):
        """Case c's block of a union nodal vector, in the case mesh's own
        numbering."""
        a, b = int(self.node_off[c]), int(self.node_off[c + 1])
        return phi[a:b][self._node_inv[c]]

    def union_phi(self, per_case):
        """The union nodal vector of per-case vectors (case numbering)."""
        t = L.torch()
        parts = [t.as_tensor(v, dtype=t.float64, device="cuda")[t.from_numpy(r.node_perm).cuda()]
                 for v, r in zip(per_case, self.renum)]
        return t.cat(parts)

    def trial_merits(self, phi, dphi, lam, mask_b):
        """sum_free R(phi + lam_c dphi)^2 per case for the per-case step
        lengths lam (host array), at the Mach numbers of the last evaluate:
        one CUDA-graph replay (the step, the batched residual and the
        per-case reduction) and one read-back."""
        t = L.torch()
        g = self._trial
        if g is None or g["frozen"] != (self.up_fz is not None) or g["mask"] is not mask_b:
            g = self._trial = self._capture_trial(mask_b)
        g["phi_base"].copy_(phi)
        g["dphi"].copy_(dphi)
        g["lam"].copy_(t.from_numpy(np.ascontiguousarray(lam, dtype=np.float64)))
        g["graph"].replay()
        return g["merit"].cpu().numpy()

    def _capture_trial(self, mask_b):
        t = L.torch()
        n = int(self.node_off[-1])
        g = {"frozen": self.up_fz is not None, "mask": mask_b,
             "phi_base": t.zeros(n, dtype=t.float64, device="cuda"),
             "dphi": t.zeros(n, dtype=t.float64, device="cuda"),
             "lam": t.zeros(self.n_cases, dtype=t.float64, device="cuda")}

        def body():
            phi_try = g["phi_base"] + g["lam"][self.case_of_node] * g["dphi"]
            R = self.evaluate(phi_try, None, jacobian=False)
            g["merit"] = self.per_case(R.masked_fill(mask_b, 0.0), "sumsq")
            g["phi_try"] = phi_try

        # captured on a side stream with capture_begin/end directly (the
        # torch.cuda.graph context would also empty the allocator cache)
        side = t.cuda.Stream()
        side.wait_stream(t.cuda.current_stream())
        graph = t.cuda.CUDAGraph()
        with t.cuda.stream(side):
            body()  # warm-up outside the graph (allocations, lazy init)
            graph.capture_begin()
            try:
                body()
            finally:
                graph.capture_end()
        t.cuda.current_stream().wait_stream(side)
        g["graph"] = graph
        return g

    @classmethod
    def tuned(cls, meshes: Sequence[BumpMesh], machs: Sequence[float], u_inf: float = 1.0,
              orderings: Sequence[str] = ("given", "morton", "hilbert"), reps: int = 5):
        """The union in the fastest of `orderings`, each with its launch
        shapes autotuned: one residual + Jacobian evaluation at the
        freestream is timed per candidate (CUDA events, median of reps).
        The report lands in ``.tuning_report``."""
        t = L.require_cuda()
        best, best_ms, report = None, None, {}
        for o in orderings:
            b = cls(meshes, u_inf=u_inf, ordering=o, tune=False)
            phi = b.ws.freestream.clone()
            b.evaluate(phi, machs, jacobian=True)
            shapes = b.ws.ev.mesh.autotune(phi, FlowParams(m_inf=float(np.min(machs)), u_inf=u_inf), reps=reps)
            ms = []
            for _ in range(reps):
                e0, e1 = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
                e0.record()
                b.evaluate(phi, machs, jacobian=True)
                e1.record()
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
            med = float(np.median(ms))
            report[o] = {"ms": med, "shapes": shapes}
            if best is None or med < best_ms:
                best, best_ms = b, med
            else:
                del b
        best.tuning_report = {"ordering": best.ordering, "candidates": report}
        return best

    def per_case(self, v, op: str):
        """Per-case max |v| ("amax") or sum v^2 ("sumsq") over the nodes."""
        t = L.torch()
        out = t.zeros(self.n_cases, dtype=t.float64, device=v.device)
        if op == "amax":
            return out.scatter_reduce(0, self.case_of_node, v.abs(), reduce="amax", include_self=True)
        return out.index_add(0, self.case_of_node, v * v)


def solve_newton_batched(batch: BatchedChannels, machs: Sequence[float], m_start: float = 0.70,
                         dm: float = 0.05, tol_residual: float = 1e-10, n_newton_max: int = 30,
                         n_picard_seed: int = 5, amg_rebuild_every: int = 2, gmres_restart: int = 60,
                         gmres_maxiter: int = 10, freeze_tol: float = 1e-6, freeze_refresh_max: int = 2,
                         use_graphs: bool = True, compact_fraction: float = 0.0,
                         verbose: bool = False) -> Dict[str, object]:
    """Lockstep Newton of every case (module docstring); returns the union
    potential, per-case convergence, iteration counts and timings.  With
    use_graphs the line search's trial evaluations replay one captured CUDA
    graph (step, batched residual, per-case merit).

    Compaction: every Krylov step, V-cycle and evaluation runs over the
    whole union, so once the cases still being solved hold less than
    `compact_fraction` of the union's elements (the others converged at
    their target Mach, or failed), the solve continues on a new union of
    those cases alone -- their potentials, frozen selections and per-case
    state carried over, the AMG hierarchy rebuilt -- and the finished
    cases' potentials are kept aside (0, the default, disables it: on the
    48-case set of 27 M tets rebuilding the union cost more than the
    smaller union saved)."""
    t = L.require_cuda()
    batch0 = batch
    ws = batch.ws
    machs = np.asarray(machs, dtype=np.float64)
    C = batch.n_cases
    C0 = C
    mask_b = ws.mask.bool()
    orig = np.arange(C)                                  # current case -> caller's case
    tets = np.array([m.n_tets for m in batch.meshes], dtype=np.int64)
    final = {"phi": [None] * C0, "converged_at": np.full(C0, -1.0), "converged_s": np.full(C0, np.nan),
             "failed": np.zeros(C0, dtype=bool), "n_newton": np.zeros(C0, dtype=np.int64),
             "froze": np.zeros(C0, dtype=bool)}
    n_compactions = 0

    def clock():
        t.cuda.synchronize()
        return time.perf_counter()

    timings = {"seed": 0.0, "residual": 0.0, "assembly": 0.0, "precond": 0.0, "linsolve": 0.0,
               "line_search": 0.0, "compaction": 0.0}
    t0 = clock()
    levels = sorted(set(mach_schedule(float(machs.max()), min(m_start, float(machs.max())), dm)))
    converged_at = np.full(C, -1.0)
    converged_s = np.full(C, np.nan)
    failed = np.zeros(C, dtype=bool)
    frozen = np.zeros(C, dtype=bool)
    n_refresh = np.zeros(C, dtype=np.int64)
    prev_live = np.full(C, np.nan)
    n_newton = np.zeros(C, dtype=np.int64)
    n_gmres_total = 0
    phi = ws.freestream.clone()
    M_pre = None
    case_node = batch.case_of_node

    # Picard seed at the first level's Mach (A(rho~(phi)) phi = b, all cases)
    m_level = np.minimum(machs, levels[0])
    for _ in range(n_picard_seed):
        batch.evaluate(phi, m_level, jacobian=False)
        A = ws.op.assemble_matrix(ws.ev.rho_tilde)
        rhs = -A.matvec(ws.phi_dir)
        rhs[ws.dn] = 0.0
        Af = with_dirichlet(A, ws.mask)
        ws.amg = M_pre = amg_for(Af, getattr(ws, "amg", None))
        x, _, _ = solve_cg(Af, rhs, M=M_pre, rtol=1e-7, maxiter=2000,
                           x0=t.where(ws.free, phi, t.zeros_like(phi)))
        phi = t.where(ws.free, x, ws.phi_dir)
    t_seed = clock() - t0
    timings["seed"] = t_seed

    for lvl, m_lev in enumerate(levels):
        m_level = np.minimum(machs, m_lev)
        # cases already converged at their target stay put; the others start
        # the level live (each level is a fresh Newton solve)
        active = ~failed & ~((converged_at >= 0) & (m_level == machs))
        batch.unfreeze(np.nonzero(active)[0])
        frozen &= ~active
        n_refresh[active] = 0
        prev_live[active] = np.nan
        history = []
        eta_prev = None
        for it in range(n_newton_max):
            finished = failed | (converged_at >= 0)
            if (compact_fraction > 0.0 and finished.any() and not finished.all()
                    and tets[~finished].sum() < compact_fraction * tets.sum()):
                tq = clock()
                keep = np.nonzero(~finished)[0]
                for c in np.nonzero(finished)[0]:
                    o = orig[c]
                    final["phi"][o] = batch.case_phi(phi, c).clone()
                    final["converged_at"][o], final["converged_s"][o] = converged_at[c], converged_s[c]
                    final["failed"][o], final["n_newton"][o], final["froze"][o] = failed[c], n_newton[c], frozen[c]
                batch, phi = _compacted(batch, phi, keep)
                ws = batch.ws
                mask_b = ws.mask.bool()
                case_node = batch.case_of_node
                M_pre = None
                machs, m_level, active = machs[keep], m_level[keep], active[keep]
                converged_at, converged_s, failed = converged_at[keep], converged_s[keep], failed[keep]
                frozen, n_refresh, prev_live = frozen[keep], n_refresh[keep], prev_live[keep]
                n_newton, orig, tets = n_newton[keep], orig[keep], tets[keep]
                history = [h[keep] for h in history]
                C = len(keep)
                n_compactions += 1
                timings["compaction"] += clock() - tq
            ta = clock()
            R = batch.evaluate(phi, m_level, jacobian=False)
            Rf = R.masked_fill(mask_b, 0.0)
            r_case = batch.per_case(Rf, "amax").cpu().numpy()
            merit = batch.per_case(Rf, "sumsq")
            history.append(r_case.copy())
            done = r_case < tol_residual
            # frozen convergence: check the live residual; refreeze there (at
            # most freeze_refresh_max times) while it has not converged and
            # still improves, as the plain driver does
            fdone = np.nonzero(active & done & frozen)[0]
            if len(fdone):
                batch.unfreeze(fdone)
                R_live = batch.evaluate(phi, m_level, jacobian=False)
                r_live = batch.per_case(R_live.masked_fill(mask_b, 0.0), "amax").cpu().numpy()
                refreeze = [c for c in fdone if r_live[c] >= tol_residual and n_refresh[c] < freeze_refresh_max
                            and (np.isnan(prev_live[c]) or r_live[c] <= 0.5 * prev_live[c])]
                for c in refreeze:
                    n_refresh[c] += 1
                    prev_live[c] = r_live[c]
                    done[c] = False
                accepted_frozen = [c for c in fdone if c not in refreeze]
                batch.freeze(refreeze)  # the state of the live evaluation just made
                batch.freeze(accepted_frozen)
                if refreeze:
                    R = batch.evaluate(phi, m_level, jacobian=False)
                    Rf = R.masked_fill(mask_b, 0.0)
                    r_case = batch.per_case(Rf, "amax").cpu().numpy()
                    merit = batch.per_case(Rf, "sumsq")
            for c in np.nonzero(active & done)[0]:
                if m_level[c] == machs[c]:
                    converged_at[c] = m_level[c]
                    converged_s[c] = time.perf_counter() - t0
            active = active & ~done
            if not active.any():
                break
            # frozen finish, case by case
            stalled = np.zeros(C, dtype=bool)
            if len(history) >= 7:
                # the plain driver's stall test: no progress over six steps
                prev_min = np.min(np.array(history[-7:-1]), axis=0)
                stalled = (r_case < 1e-3) & (r_case > 0.25 * prev_min) & (r_case < 2.0 * prev_min)
            to_freeze = active & ~frozen & ((r_case < freeze_tol) | stalled)
            if to_freeze.any():
                batch.freeze(np.nonzero(to_freeze)[0])
                frozen |= to_freeze
                R = batch.evaluate(phi, m_level, jacobian=False)
                Rf = R.masked_fill(mask_b, 0.0)
                merit = batch.per_case(Rf, "sumsq")
            tb = clock()
            timings["residual"] += tb - ta
            batch.evaluate(phi, m_level, jacobian=True)
            J = with_dirichlet(ws.ev.jacobian(), ws.mask)
            tc = clock()
            timings["assembly"] += tc - tb
            if M_pre is None or it % amg_rebuild_every == 0:
                ws.amg = M_pre = amg_for(ws.picard_matrix(), getattr(ws, "amg", None))
            td = clock()
            timings["precond"] += td - tc
            r_act = r_case[active]
            r_prev = history[-2][active] if len(history) > 1 else None
            etas = [_ew_forcing(float(a), None if r_prev is None else float(b), eta_prev)
                    for a, b in zip(r_act, r_prev if r_prev is not None else [None] * len(r_act))]
            eta = min(etas)
            eta_prev = eta
            act_node = t.from_numpy(active).cuda()[case_node]
            # each case's block of the right-hand side scaled to unit norm, so
            # that the joint Krylov residual weighs the cases equally (the
            # Jacobian is block diagonal: the scaling comes back out exactly)
            scale = t.sqrt(merit).clamp_min(1e-300)
            rhs = (-Rf / scale[case_node]).masked_fill(~act_node, 0.0)
            y, n_it, _ = solve_gmres(J, rhs, M=M_pre, rtol=eta / np.sqrt(active.sum()),
                                     restart=gmres_restart, maxiter=gmres_maxiter, on_fail="return")
            dphi = y * scale[case_node]
            te = clock()
            timings["linsolve"] += te - td
            n_gmres_total += n_it
            n_newton[active] += 1
            dphi = dphi.masked_fill(mask_b | ~act_node, 0.0)
            # per-case backtracking: lam halves for the cases whose merit rose
            lam = np.where(active, 1.0, 0.0)
            accepted = ~active
            best_lam = np.zeros(C)
            best_merit = np.full(C, np.inf)
            merit_h = merit.cpu().numpy()
            for _ in range(5):
                if use_graphs:
                    m_try = batch.trial_merits(phi, dphi, lam, mask_b)
                else:
                    lam_node = t.from_numpy(lam).cuda()[case_node]
                    phi_try = phi + lam_node * dphi
                    R_try = batch.evaluate(phi_try, m_level, jacobian=False)
                    m_try = batch.per_case(R_try.masked_fill(mask_b, 0.0), "sumsq").cpu().numpy()
                ok = np.isfinite(m_try) & (m_try <= merit_h) & ~accepted
                better = np.isfinite(m_try) & (m_try < best_merit) & ~accepted
                best_lam[better] = lam[better]
                best_merit[better] = m_try[better]
                accepted |= ok
                if accepted.all():
                    break
                lam = np.where(accepted, lam, 0.5 * lam)
            lam = np.where(accepted, lam, best_lam)
            phi = phi + t.from_numpy(lam).cuda()[case_node] * dphi
            timings["line_search"] += clock() - te
            if verbose:
                print(f"  level M<={m_lev:.3f} it {it}: max|R| active = {r_act.max():.3e}")
        # a case still active at the end of a level failed it
        failed |= active
    t_total = clock() - t0
    for c in range(C):
        o = orig[c]
        final["phi"][o] = batch.case_phi(phi, c)
        final["converged_at"][o], final["converged_s"][o] = converged_at[c], converged_s[c]
        final["failed"][o], final["n_newton"][o], final["froze"][o] = failed[c], n_newton[c], frozen[c]
    phi_union = phi if batch is batch0 else batch0.union_phi(final["phi"])
    return {"phi": phi_union, "converged": final["converged_at"] >= 0, "failed": final["failed"],
            "n_newton": final["n_newton"], "n_gmres_total": n_gmres_total, "levels": levels, "time_s": t_total,
            "seed_s": t_seed, "timings": timings, "n_compactions": n_compactions,
            "converged_s": final["converged_s"], "froze": final["froze"]}


def _compacted(batch: BatchedChannels, phi, keep):
    """A new union of the cases `keep` of `batch` (same ordering and launch
    shapes), with their potentials and frozen selections carried over."""
    t = L.torch()
    new = BatchedChannels([batch.meshes[c] for c in keep], u_inf=batch.u_inf, ordering=batch.ordering,
                          tune=False)
    tu = batch.ws.ev.mesh.tuning()
    new.ws.ev.mesh.set_tuning(tu["elem_persistent"], tu["elem_threads_per_sm"], tu["row_lanes"], tu["row_plan8"],
                              tu["assembly"], tu["tile_elems"], tu["tile_stretch"])
    if tu["assembly"] == 1:
        new.ws.ev.mesh.tile_info()
    phi_new = new.union_phi([batch.case_phi(phi, c) for c in keep])
    if batch.up_fz is not None:
        new.up_fz = t.zeros(new.n_tets, dtype=t.int64, device="cuda")
        new.br_fz = t.full((new.n_tets,), -1, dtype=t.int8, device="cuda")
        for k, c in enumerate(keep):
            a, b = int(batch.elem_off[c]), int(batch.elem_off[c + 1])
            na, nb = int(new.elem_off[k]), int(new.elem_off[k + 1])
            new.up_fz[na:nb] = batch.up_fz[a:b] - a + na
            new.br_fz[na:nb] = batch.br_fz[a:b]
    return new, phi_new


class CaseSet:
    """Independent channel cases solved on one device, each where it runs
    fastest: the cases below ``batch_below`` tets share one lockstep union
    (``BatchedChannels``: their launches, V-cycles and host synchronisations
    are shared, which is where a small case spends its time), the larger
    cases run one by one through the plain driver (a case of that size
    fills the GPU alone, and lockstep would only tie it to the slowest
    case's iteration count).  Everything the solves reuse -- the union, its
    launch shapes, the per-case workspaces -- is built here, so ``solve``
    times the solves alone."""

    def __init__(self, meshes: Sequence[BumpMesh], machs: Sequence[float], batch_below: int = 300_000,
                 u_inf: float = 1.0, tune_orderings: Sequence[str] = ("given",)):
        L.require_cuda()
        self.meshes = list(meshes)
        self.machs = np.asarray(machs, dtype=np.float64)
        if len(self.machs) != len(self.meshes):
            raise ValueError(f"{len(self.meshes)} meshes but {len(self.machs)} Mach numbers")
        tets = np.array([m.n_tets for m in self.meshes], dtype=np.int64)
        small = np.nonzero(tets < batch_below)[0]
        if len(small) < 2:
            small = np.zeros(0, dtype=np.int64)
        self.small = small
        self.large = np.setdiff1d(np.arange(len(self.meshes)), small)
        self.batch = None
        self.batch_tuning = None
        if len(small):
            self.batch = BatchedChannels.tuned([self.meshes[c] for c in small], self.machs[small], u_inf=u_inf,
                                               orderings=tune_orderings)
            self.batch_tuning = self.batch.ws.ev.mesh.tuning()
        self.wss = {int(c): ChannelWorkspace(self.meshes[c].nodes, self.meshes[c].elements,
                                             self.meshes[c].dirichlet_nodes, u_inf=u_inf) for c in self.large}

    def solve(self, m_start: float = 0.70, dm: float = 0.05, tol_residual: float = 1e-10,
              batched_kw: Optional[dict] = None, plain_kw: Optional[dict] = None) -> Dict[str, object]:
        """Every case to |R_free|_inf < tol_residual at its Mach number:
        the union first, then the large cases.  Returns per-case potentials
        (case numbering, device), convergence, Newton steps and the time at
        which each case finished (seconds from the start), and the wall
        time with the device synchronised."""
        t = L.require_cuda()
        from .newton import solve_newton_transonic
        C = len(self.meshes)
        out = {"phi": [None] * C, "converged": np.zeros(C, dtype=bool), "n_newton": np.zeros(C, dtype=np.int64),
               "case_s": np.full(C, np.nan), "n_batched": int(len(self.small)), "n_plain": int(len(self.large))}
        t.cuda.synchronize()
        t0 = time.perf_counter()
        if self.batch is not None:
            res = solve_newton_batched(self.batch, self.machs[self.small], m_start=m_start, dm=dm,
                                       tol_residual=tol_residual, compact_fraction=0.0, **(batched_kw or {}))
            for k, c in enumerate(self.small):
                out["phi"][c] = self.batch.case_phi(res["phi"], k)
                out["converged"][c] = bool(res["converged"][k])
                out["n_newton"][c] = int(res["n_newton"][k])
                out["case_s"][c] = res["converged_s"][k]
            out["batched_timings"] = res["timings"]
            out["batched_s"] = res["time_s"]
        for c in self.large:
            M = float(self.machs[c])
            r = solve_newton_transonic(self.wss[int(c)], M, m_start=min(m_start, M), dm=dm,
                                       tol_residual=tol_residual, **(plain_kw or {}))
            out["phi"][c] = r["phi"]
            out["converged"][c] = bool(r["converged"])
            out["n_newton"][c] = int(sum(lv[1] for lv in r["level_history"]))
            t.cuda.synchronize()
            out["case_s"][c] = time.perf_counter() - t0
        t.cuda.synchronize()
        out["time_s"] = time.perf_counter() - t0
        return out
