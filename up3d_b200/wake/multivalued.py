"""Extended-DOF (multivalued) operator of the level-set wake on the B200,
with the reference's interface (pyfp3d/wake/multivalued.py:43-907).

Each node of a cut element carries an aux DOF holding the potential on the
other side of the sheet.  The operator is the ordinary P1 operator plus
corrections on the cut elements:

* assemble_matrix: the device P1 matrix (PicardOperator.assemble_matrix)
  folded into an extended CSR whose pattern is planned once per closure --
  the union of the P1 pattern and the correction triplets, with the slot of
  every P1 entry and every correction fixed -- plus the cut-element
  corrections (kernels.cut_assembly: redirection + weld rows, or the
  two-sided mass conservation + wake least squares), formed on the host
  over the few cut elements, summed per slot in the reference's triplet
  order and added on the device;
* element_rho_tilde / newton_side_data / freeze_side_state: the walk flux
  once per side, on that side's potential and on a face graph restricted to
  that side's elements (UpwindOperator.face_neighbors on a forked mesh
  handle), everything on the device.

Not built: the pressure Kutta rows at TE nodes (te_kutta="pressure" when
the map has TE nodes), the tip taper and the span blend; each raises
NotImplementedError.  The cut census itself is wake.cut_elements.
"""

from __future__ import annotations

from typing import Optional

import numpy as np

from .. import _lib as L
from ..kernels import cut_assembly as ca
from ..kernels.jacobian import PicardOperator
from ..mesh.device import DeviceCSR


def _np(x):
    return x.detach().cpu().numpy() if L.is_torch(x) else np.asarray(x)


class _ExtendedPattern:
    """The extended CSR of one closure: the P1 pattern (rows < n_main) and
    the correction triplets' (row, col) pairs, planned once."""

    def __init__(self, n_total, base_indptr, base_indices, rows, cols):
        t = L.torch()
        n_main = len(base_indptr) - 1
        base_rows = np.repeat(np.arange(n_main, dtype=np.int64), np.diff(base_indptr))
        key_base = base_rows * n_total + base_indices.astype(np.int64)
        key_corr = rows.astype(np.int64) * n_total + cols.astype(np.int64)
        keys = np.unique(np.concatenate([key_base, key_corr]))
        self.n_total, self.nnz = n_total, len(keys)
        ext_rows = keys // n_total
        indptr = np.zeros(n_total + 1, dtype=np.int64)
        np.add.at(indptr, ext_rows + 1, 1)
        indptr = np.cumsum(indptr)
        self.indptr = L.to_device(indptr.astype(np.int32), t.int32)
        self.indices = L.to_device((keys % n_total).astype(np.int32), t.int32)
        self.base_slot = L.to_device(np.searchsorted(keys, key_base), t.int64)
        corr_slot = np.searchsorted(keys, key_corr)
        self.corr_slots, self.corr_inv = np.unique(corr_slot, return_inverse=True)
        self.corr_slots_d = L.to_device(self.corr_slots, t.int64)

    def assemble(self, base_data, corr_values) -> DeviceCSR:
        """P1 values into their slots, then each correction slot's sum (in
        triplet order) added."""
        t = L.torch()
        data = t.zeros(self.nnz, dtype=t.float64, device="cuda")
        data[self.base_slot] = base_data
        if len(self.corr_slots):
            tot = np.bincount(self.corr_inv, weights=corr_values, minlength=len(self.corr_slots))
            data[self.corr_slots_d] += L.to_device(tot, t.float64)
        return DeviceCSR(self.indptr, self.indices, data, (self.n_total, self.n_total))


class MultivaluedOperator:
    """Extended-DOF assembly and per-side densities on a cut mesh (module
    docstring).  nodes, elements: the mesh; cm: its CutElementMap
    (wake.cut_elements, or the reference's -- the same attributes);
    levelset: the WakeLevelSet, needed for the wake least-squares closure."""

    def __init__(self, nodes, elements, cm, levelset=None, span_blend=None):
        t = L.require_cuda()
        if span_blend is not None:
            raise NotImplementedError("span_blend (the spanwise termination blend of the wake rows) is not built")
        self.nodes = np.ascontiguousarray(_np(nodes), dtype=np.float64)
        el = np.ascontiguousarray(_np(elements), dtype=np.int64)
        self.op = PicardOperator(t.as_tensor(self.nodes, device="cuda"), t.as_tensor(el.astype(np.int32), device="cuda"))
        self.elements = el
        self.cm = cm
        self.levelset = levelset
        self.n_main = cm.n_main
        self.n_ext = cm.n_ext_dofs
        self.n_total = cm.n_total_dofs
        if self.op.n_nodes != self.n_main:
            raise ValueError("CutElementMap.n_main != mesh node count -- the map was built on a different mesh")
        E = self.op.n_tets
        self.plain, self._special = ca.special_elements(cm, E)
        self._special_ids = np.flatnonzero(self._special)
        B, V = self.op.mesh.geometry()
        ids = L.to_device(self._special_ids, t.int64)
        self._Bs, self._Vs = B[ids].cpu().numpy(), V[ids].cpu().numpy()
        self._sidx = np.full(E, -1, dtype=np.int64)
        self._sidx[self._special_ids] = np.arange(len(self._special_ids))
        self._closure_coo = ca.continuity_closure_coo(cm)
        self._nonte_rows = ca.nonte_aux_rows(cm)
        self._ls_coo = None
        if levelset is not None and len(cm.cut_elems):
            cen = self.nodes[el[cm.cut_elems]].mean(axis=1)
            self._ls_coo = ca.wake_ls_coo(self, cm, levelset.surface_normals(cen), levelset.direction)
        self._patterns = {}
        self._side_sets = self._side_upw = self._side_dof = self._side_read = self._mixed_plain = None
        self._elem_plus = None
        self.nu_max, self.n_nu_active, self.n_floored, self.n_limited = 0.0, 0, 0, 0
        self._nu_active = np.zeros(E, dtype=bool)
        self.n_span_blended = 0

    # ------------------------------------------------------------ geometry

    def cut_geometry(self, ids):
        """B and V (host) of special elements (cut or below-TE fan)."""
        k = self._sidx[np.asarray(ids, dtype=np.int64)]
        if np.any(k < 0):
            raise ValueError("cut_geometry is kept for the cut and below-TE-fan elements only")
        return self._Bs[k], self._Vs[k]

    @property
    def B(self):
        return self.op.B

    @property
    def V(self):
        return self.op.V

    def _pattern(self, key, rows, cols):
        p = self._patterns.get(key)
        if p is None:
            m = self.op.mesh
            p = self._patterns[key] = _ExtendedPattern(self.n_total, m.indptr.cpu().numpy(), m.indices.cpu().numpy(),
                                                       rows, cols)
        return p

    # ------------------------------------------------------------ assembly

    def assemble_matrix(self, rho_tilde=None, closure: str = "continuity", te_kutta: str = "pressure",
                        phi_ext=None, tip_taper=None) -> DeviceCSR:
        """Extended (n_total x n_total) matrix (wake/multivalued.py:276-381)
        as a DeviceCSR (``to_scipy()`` for the host copy)."""
        t = L.torch()
        cm = self.cm
        if tip_taper is not None and not np.all(np.asarray(tip_taper) == 1.0):
            raise NotImplementedError("tip_taper (the TE weld blend of the pressure Kutta rows) is not built")
        if closure == "continuity":
            base = self.op.assemble_matrix(None if rho_tilde is None else L.to_device(rho_tilde, t.float64))
            r = ca.multivalued_redirection_coo(self, cm, rho_tilde)
            c = self._closure_coo
            rows, cols, vals = (np.concatenate([r[i], c[i]]) for i in range(3))
            key = "continuity"
        elif closure == "wake_ls":
            if self._ls_coo is None:
                raise ValueError("wake_ls closure needs a WakeLevelSet (pass levelset= to MultivaluedOperator) "
                                 "and a non-empty cut set")
            if te_kutta == "pressure" and len(cm.te_nodes):
                raise NotImplementedError("te_kutta='pressure' (the TE pressure-equality rows) is not built; "
                                          "te_kutta='mass' keeps mass conservation on the TE aux rows")
            if te_kutta not in ("pressure", "mass"):
                raise NotImplementedError(f"te_kutta={te_kutta!r} unknown")
            rho_up, rho_lo = (None, None) if rho_tilde is None else rho_tilde
            E = self.op.n_tets
            if rho_up is None:
                ru = rl = t.ones(E, dtype=t.float64, device="cuda")
            else:
                ru, rl = L.to_device(rho_up, t.float64), L.to_device(rho_lo, t.float64)
            plus = L.to_device(self._plain_plus(), t.bool)
            w = t.where(plus, ru, rl)
            w[L.to_device(self._special_ids, t.int64)] = 0.0     # special elements: corrections
            base = self.op.assemble_matrix(w)
            m = ca.mass_conservation_coo(self, cm, None if rho_up is None else _np(ru),
                                         None if rho_up is None else _np(rl), elements="special")
            drop = np.zeros(self.n_total, dtype=bool)
            drop[self._nonte_rows] = True
            keep = ~drop[m[0]]
            ls = self._ls_coo
            rows, cols, vals = (np.concatenate([m[i][keep], ls[i]]) for i in range(3))
            key = "wake_ls"
        else:
            raise NotImplementedError(f"closure={closure!r} unknown")
        pat = self._pattern(key, rows, cols)
        return pat.assemble(base.data, vals)

    def _plain_plus(self):
        """(E,) bool: a plain element on the "+" side (max node side +1)."""
        return self.cm.node_side[self.elements].max(axis=1) == 1

    # ------------------------------------------------------------ DOF bookkeeping

    def main_potential(self, phi_ext):
        return phi_ext[: self.n_main]

    def te_jump(self, phi_ext):
        return self.node_jump(phi_ext, self.cm.te_nodes)

    def node_jump(self, phi_ext, node_ids):
        """side * (main - aux) at the given nodes (0 at nodes without an aux
        DOF)."""
        host = not L.is_torch(phi_ext)
        p = np.asarray(_np(phi_ext), dtype=np.float64)
        node_ids = np.asarray(node_ids, dtype=np.int64)
        aux = self.cm.ext_dof_of_node[node_ids]
        has = aux >= 0
        out = np.zeros(len(node_ids))
        j = node_ids[has]
        out[has] = self.cm.node_side[j] * (p[j] - p[aux[has]])
        return out if host else L.to_device(out, L.torch().float64)

    def side_potentials(self, phi_ext):
        """(phi_upper, phi_lower) nodal fields: at a cut node the own side is
        the main DOF and the other side the aux DOF."""
        t = L.torch()
        host = not L.is_torch(phi_ext)
        p = L.to_device(phi_ext, t.float64)
        up, lo = p[: self.n_main].clone(), p[: self.n_main].clone()
        cut_nodes = np.flatnonzero(self.cm.ext_dof_of_node >= 0)
        aux = self.cm.ext_dof_of_node[cut_nodes]
        plus = self.cm.node_side[cut_nodes] == 1
        lo[L.to_device(cut_nodes[plus], t.int64)] = p[L.to_device(aux[plus], t.int64)]
        up[L.to_device(cut_nodes[~plus], t.int64)] = p[L.to_device(aux[~plus], t.int64)]
        return (up.cpu().numpy(), lo.cpu().numpy()) if host else (up, lo)

    # ------------------------------------------------------------ per-side densities

    def _side_element_sets(self):
        """(in_upper, in_lower) host masks: plain "+" and cut elements carry
        an upper copy; plain "-", cut and below-TE-fan elements a lower one."""
        if self._side_sets is None:
            E = self.op.n_tets
            cut = np.zeros(E, dtype=bool)
            cut[self.cm.cut_elems] = True
            tel = np.zeros(E, dtype=bool)
            tel[self.cm.te_lower_elems] = True
            plain = ~cut & ~tel
            plus = plain & self._plain_plus()
            self._side_sets = (plus | cut, (plain & ~plus) | cut | tel)
        return self._side_sets

    def _side_upwind(self):
        """Two walk-flux operators whose face graphs keep only faces between
        elements of their own side (wake/multivalued.py:439-470)."""
        if self._side_upw is None:
            from ..kernels.upwind import UpwindOperator
            t = L.torch()
            fn0 = self.op.mesh.face_neighbors().to(t.int64)
            ops = []
            for keep in self._side_element_sets():
                k = L.to_device(keep, t.bool)
                ok = (fn0 >= 0) & k[fn0.clamp_min(0)] & k[:, None]
                fn = t.where(ok, fn0, t.full_like(fn0, -1)).to(t.int32).contiguous()
                upw = UpwindOperator(t.as_tensor(self.nodes, device="cuda"),
                                     t.as_tensor(self.elements.astype(np.int32), device="cuda"), mesh=self.op.mesh)
                upw.face_neighbors = fn
                ops.append(upw)
            self._side_upw = tuple(ops)
        return self._side_upw

    def _mixed_plain_mask(self):
        """Plain elements whose nodes straddle the level set."""
        if self._mixed_plain is None:
            side = self.cm.node_side[self.elements]
            self._mixed_plain = ~self._special & (side.min(axis=1) != side.max(axis=1))
        return self._mixed_plain

    def _apply_main_density(self, phi_ext_d, grad, q2):
        """A mixed-side plain element reads its gradient and q^2 from the
        main field (wake/multivalued.py:543-579)."""
        t = L.torch()
        mask = self._mixed_plain_mask()
        if not mask.any():
            return grad, q2
        grad, q2 = grad.clone(), q2.clone()
        gm, qm = self.op.velocities(phi_ext_d[: self.n_main].contiguous())
        md = L.to_device(mask, t.bool)
        grad[md] = gm[md]
        q2[md] = qm[md]
        return grad, q2

    def _side_fields(self, phi_ext_d, m_inf, gamma_air, u_inf, m_cap):
        """Per side: (phi_s, grad, q2n, q2l, rho) on the device."""
        from ..physics.isentropic import density_field, limit_q2_field
        out = []
        for phi_s in self.side_potentials(phi_ext_d):
            grad, q2 = self.op.velocities(phi_s)
            grad, q2 = self._apply_main_density(phi_ext_d, grad.clone(), q2.clone())
            q2n = q2 / u_inf ** 2
            q2l = limit_q2_field(q2n, m_inf, m_cap, gamma_air)
            out.append((phi_s, grad, q2n, q2l, density_field(q2l, m_inf, gamma_air)))
        return out

    def _monitors(self, nus, keeps, floored, limited):
        t = L.torch()
        own = t.cat([nu[k] for nu, k in zip(nus, keeps)])
        self.nu_max = float(own.max()) if own.numel() else 0.0
        self.n_nu_active = int((own > 0.0).sum())
        self.n_floored = floored
        self.n_limited = limited
        act = t.zeros_like(keeps[0])
        for nu, k in zip(nus, keeps):
            act |= (nu > 0.0) & k
        self._nu_active = act.cpu().numpy()

    def element_rho_tilde(self, phi_ext, m_inf, upwind_c, m_crit, gamma_air=1.4, u_inf=1.0, m_cap=3.0,
                          rho_floor=0.05):
        """(rho_tilde_upper, rho_tilde_lower): the walk flux of each side on
        its own field and own-side face graph, speed limiter per side
        (wake/multivalued.py:472-524).  Refreshes the own-side monitors
        nu_max, n_nu_active, n_floored, n_limited."""
        t = L.require_cuda()
        host = not L.is_torch(phi_ext)
        p = L.to_device(phi_ext, t.float64)
        keeps = [L.to_device(k, t.bool) for k in self._side_element_sets()]
        out, nus, floored, limited = [], [], 0, 0
        for (phi_s, grad, q2n, q2l, rho), upw, keep in zip(self._side_fields(p, m_inf, gamma_air, u_inf, m_cap),
                                                           self._side_upwind(), keeps):
            limited += int(((q2l != q2n) & keep).sum())
            rt = upw.rho_tilde(grad, q2l, rho, m_inf, upwind_c, m_crit, gamma_air, rho_floor).clone()
            nus.append(upw.nu.clone())
            floored += int(((rt == rho_floor) & keep).sum())
            out.append(rt)
        self._monitors(nus, keeps, floored, limited)
        return tuple(o.cpu().numpy() for o in out) if host else tuple(out)

    def nu_active_elements(self):
        return np.flatnonzero(self._nu_active)

    def element_densities(self, phi_ext, m_inf, gamma_air=1.4, u_inf=1.0):
        """(rho_upper, rho_lower) of the two side fields (no upwinding), each
        valid on its own side's elements (wake/multivalued.py:797-819)."""
        from ..physics.isentropic import density_field
        t = L.require_cuda()
        host = not L.is_torch(phi_ext)
        p = L.to_device(phi_ext, t.float64)
        out = []
        for phi_s in self.side_potentials(p):
            grad, q2 = self.op.velocities(phi_s)
            _, q2 = self._apply_main_density(p, grad.clone(), q2.clone())
            out.append(density_field(q2 / u_inf ** 2, m_inf, gamma_air).clone())
        return tuple(o.cpu().numpy() for o in out) if host else tuple(out)

    def own_side_field(self, field_up, field_lo):
        """Each element's own-side value: upper on "+" plain and cut
        elements, lower elsewhere."""
        if self._elem_plus is None:
            self._elem_plus = self._side_element_sets()[0]
        if L.is_torch(field_up):
            t = L.torch()
            return t.where(L.to_device(self._elem_plus, t.bool), field_up, field_lo)
        return np.where(self._elem_plus, field_up, field_lo)

    def element_mach2(self, phi_ext, m_inf, gamma_air=1.4, u_inf=1.0, mixed_plain="main"):
        """Own-side element M^2, the larger side on cut elements; mixed-side
        plain elements from the main field ("main") or the side fields
        ("side") (wake/multivalued.py:842-895)."""
        from ..physics.isentropic import mach_squared_field
        t = L.require_cuda()
        if mixed_plain not in ("main", "side"):
            raise ValueError(f"mixed_plain={mixed_plain!r} unknown")
        host = not L.is_torch(phi_ext)
        p = L.to_device(phi_ext, t.float64)
        m2s = []
        for phi_s in self.side_potentials(p):
            _, q2 = self.op.velocities(phi_s)
            m2s.append(mach_squared_field(q2 / u_inf ** 2, m_inf, gamma_air).clone())
        m2 = self.own_side_field(m2s[0], m2s[1])
        cut = L.to_device(np.asarray(self.cm.cut_elems, dtype=np.int64), t.int64)
        m2[cut] = t.maximum(m2s[0][cut], m2s[1][cut])
        if mixed_plain == "main" and self._mixed_plain_mask().any():
            _, qm = self.op.velocities(p[: self.n_main].contiguous())
            fix = L.to_device(self._mixed_plain_mask(), t.bool)
            m2[fix] = mach_squared_field(qm / u_inf ** 2, m_inf, gamma_air)[fix]
        return m2.cpu().numpy() if host else m2

    # ------------------------------------------------------------ per-side Newton records

    def _side_dofvecs(self):
        """(dof_upper, dof_lower) (E, 4): the DOF vectors each element's copy
        scatters with (wake/multivalued.py:630-658)."""
        if self._side_dof is None:
            cm, el = self.cm, self.elements
            te = np.zeros(cm.n_main, dtype=bool)
            te[cm.te_nodes] = True
            du, dl = el.copy(), el.copy()
            du[cm.cut_elems] = cm.dofs_upper
            dl[cm.cut_elems] = cm.dofs_lower
            tel = np.asarray(cm.te_lower_elems, dtype=np.int64)
            if len(tel):
                dl[tel] = np.where(te[el[tel]], cm.ext_dof_of_node[el[tel]], el[tel])
            self._side_dof = (du, dl)
        return self._side_dof

    def _side_readvecs(self):
        """(read_upper, read_lower) (E, 4): the DOF each element node's side
        field reads; mixed-side plain elements read the main DOFs
        (wake/multivalued.py:581-628)."""
        if self._side_read is None:
            cm, el = self.cm, self.elements
            ext = cm.ext_dof_of_node[el]
            side = cm.node_side[el]
            has = ext >= 0
            ru = np.where((side == 1) | ~has, el, ext)
            rl = np.where((side == -1) | ~has, el, ext)
            mp = self._mixed_plain_mask()
            ru[mp] = el[mp]
            rl[mp] = el[mp]
            if len(cm.cut_elems) and not (np.array_equal(ru[cm.cut_elems], cm.dofs_upper)
                                          and np.array_equal(rl[cm.cut_elems], cm.dofs_lower)):
                raise RuntimeError("side read map differs from the cut elements' DOF vectors")
            self._side_read = (ru, rl)
        return self._side_read

    def newton_side_data(self, phi_ext, m_inf, upwind_c, m_crit, gamma_air=1.4, u_inf=1.0, m_cap=3.0,
                         rho_floor=0.05, frozen=None):
        """Per side (upper, lower) the records the level-set Newton
        Jacobian needs (wake/multivalued.py:660-752): rho_tilde, s_e, s_u,
        upstream, grad, lim_mask, keep, dofvec, readvec, grad_row; live, or
        from a frozen (upstream, branch) pair per side.  Monitors as
        element_rho_tilde."""
        t = L.require_cuda()
        host = not L.is_torch(phi_ext)
        p = L.to_device(phi_ext, t.float64)
        keeps_h = self._side_element_sets()
        keeps = [L.to_device(k, t.bool) for k in keeps_h]
        fz = (None, None) if frozen is None else frozen
        B = self.op.mesh.geometry()[0]
        out, nus, floored, limited = [], [], 0, 0
        for (phi_s, grad, q2n, q2l, rho), upw, keep, keep_h, dof, read, f in zip(
                self._side_fields(p, m_inf, gamma_air, u_inf, m_cap), self._side_upwind(), keeps, keeps_h,
                self._side_dofvecs(), self._side_readvecs(), fz):
            lim = q2l == q2n
            limited += int(((~lim) & keep).sum())
            if f is None:
                rt = upw.rho_tilde(grad, q2l, rho, m_inf, upwind_c, m_crit, gamma_air, rho_floor).clone()
                floored += int(((rt == rho_floor) & keep).sum())
                s_e, s_u, up = upw.rho_tilde_sensitivities(grad, q2l, rho, m_inf, upwind_c, m_crit, gamma_air,
                                                           rho_floor)
                up = up.clone()
            else:
                up_sel, branch = (L.to_device(a, t.int64 if k == 0 else t.int8) for k, a in enumerate(f))
                rt = upw.rho_tilde_frozen(q2l, rho, up_sel, branch, m_inf, upwind_c, m_crit, gamma_air,
                                          rho_floor).clone()
                floored += int(((branch == 3) & keep).sum())
                s_e, s_u = upw.rho_tilde_frozen_sensitivities(q2l, rho, up_sel, branch, m_inf, upwind_c, m_crit,
                                                              gamma_air, rho_floor)
                up = up_sel
            nus.append(upw.nu.clone())
            dof_d = L.to_device(dof, t.int64)
            rec = {"rho_tilde": rt, "s_e": s_e.clone(), "s_u": s_u.clone(), "upstream": up, "grad": grad.clone(),
                   "lim_mask": lim, "keep": keep_h, "dofvec": dof, "readvec": read,
                   "grad_row": t.einsum("ek,ekd->ed", p[dof_d], B)}
            if host:
                rec = {k: (v.cpu().numpy() if L.is_torch(v) else v) for k, v in rec.items()}
            out.append(rec)
        self._monitors(nus, keeps, floored, limited)
        return out[0], out[1]

    def freeze_side_state(self, phi_ext, m_inf, upwind_c, m_crit, gamma_air=1.4, u_inf=1.0, m_cap=3.0,
                          rho_floor=0.05):
        """Per side the (upstream, branch) selection at phi_ext, for
        newton_side_data(frozen=...) (wake/multivalued.py:754-786)."""
        t = L.require_cuda()
        host = not L.is_torch(phi_ext)
        p = L.to_device(phi_ext, t.float64)
        frozen = []
        for (phi_s, grad, q2n, q2l, rho), upw in zip(self._side_fields(p, m_inf, gamma_air, u_inf, m_cap),
                                                     self._side_upwind()):
            up, br = upw.freeze_upwind_state(grad, q2l, rho, m_inf, upwind_c, m_crit, gamma_air, rho_floor)
            frozen.append((up.cpu().numpy(), br.cpu().numpy()) if host else (up.clone(), br.clone()))
        return frozen[0], frozen[1]
