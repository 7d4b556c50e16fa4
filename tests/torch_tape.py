"""Test infrastructure: the reference's binary two-phase FP64 time step
(NUMPHASES = 2, one BINARY component, isothermal) restated in float64 torch
operations, so that torch's autograd tape differentiates it.  The gradients
of a loss through a run of these steps are the independent reference for the
CUDA adjoint (gp_adjoint), which differentiates its own cell functions
forward-mode; the forward values equal the CPU oracle's bit for bit (the same
scalar operations in the same order, element by element).

It follows the oracle (oracle/gp_oracle.c) function by function, which
follows the reference:
  boundary copy            apply_boundary_conditions    boundary_serial.h:176-203
  phi faces                calculate_gradients_phasefield_2D  calculate_gradients.h:92-131
  delta-phi                calculate_divergence_phasefield_2D  calculate_divergence_phasefield.h:4-62
    interface energy       function_A_00 / A_01          function_A_00.h:4-58, function_A_01.h:4-219
    anisotropy             anisotropy_01_dAdq / _ac      anisotropy_01.h:9-48, functionQ.h:4-40
    potential              function_W_01 / W_02           functionW_01.h:6-39, functionW_02.h:4-33
    driving force          function_F_01_dpsi             functionF_01.h:41-57
    projection             projection_on_simplex          simplex_projection.h:1-49
  mu faces, fluxes         calculate_gradients_concentration_2D, calculate_fluxes_concentration_2D
                           calculate_gradients.h:132-185, calculate_fluxes_concentration.h:4-145
  concentration update     calculate_divergence_concentration_2D  calculate_divergence_concentration.h:4-153
Only the cells the interior's update reads are evaluated: the ring of
delta-phi around the interior, the faces around it; the ghost cells of the
new state are boundary copies.  Branches (active phases, the projection's
cases, the bulk test, the anti-trapping guards) are taken by value, as the
step takes them: the tape holds the derivative of the branch taken.
"""
import math

import numpy as np
import torch

from oracle_py import Oracle


def _copy_map(m, lo, hi):
    """ghosted index (m + 6 of them) -> interior index of the cell it holds:
    the boundary copy's tables (Neumann mirrors about the boundary cell,
    periodic wraps with period m-1)"""
    r = m + 6
    out = []
    for g in range(r):
        src = g
        if g < 3:
            j = 2 - g
            src = 4 + j if lo == 1 else r - 5 - j
        elif g >= r - 3:
            j = g - (r - 3)
            src = r - 5 - j if hi == 1 else 4 + j
        out.append(src - 3)
    return torch.tensor(out, dtype=torch.long)


class _Sqrt(torch.autograd.Function):
    """correctly rounded square root (numpy's, as the C library's sqrt), with
    its derivative 1/(2 sqrt x): torch's vectorised float64 sqrt can be one
    ulp off"""

    @staticmethod
    def forward(ctx, x):
        r = torch.from_numpy(np.sqrt(x.detach().cpu().numpy())).to(x.device)
        ctx.save_for_backward(r)
        return r

    @staticmethod
    def backward(ctx, g):
        (r,) = ctx.saved_tensors
        return g / (2.0 * r)


def _rot2(M, t0, t1):
    """multiply(Rotation_matrix, q, out, 2) (matrix.h:10-20): s = 0; s = s + M[i][j]*q[j]"""
    r0 = (0.0 + M[0][0] * t0) + M[0][1] * t1
    r1 = (0.0 + M[1][0] * t0) + M[1][1] * t1
    return r0, r1


class TapeStep:
    """One FP64 time step of a binary two-phase run as torch operations, with
    theta = (Tau_01, dab_01, epsilon, GAMMA_01) a float64 tensor."""

    def __init__(self, p):
        if p.numphases != 2 or p.numcomponents != 2 or not p.binary or not p.isothermal:
            raise ValueError("binary two-phase isothermal runs only")
        self.p = p
        o = Oracle(p)
        c = o.consts()
        o.close()
        self.mx, self.my = int(p.mesh_x), int(p.mesh_y)
        self.rx, self.ry = self.mx + 6, self.my + 6
        self.dx, self.dy, self.dt = float(p.deltax), float(p.deltay), float(p.deltat)
        self.aniso = p.function_anisotropy == 1
        self.well = p.function_w == 2
        self.tau_default = float(p.tau)
        self.cmu = [float(c["cmu"][b][0][0]) for b in range(2)]
        self.B = [float(c["B"][b][0]) for b in range(2)]
        self.C = [float(c["C"][b]) for b in range(2)]
        T, Teq = float(p.T), float(p.Teq)
        self.E = [float(c["Beq"][b][0]) + float(c["dBbdT"][b][0]) * (T - Teq) for b in range(2)]
        self.A = [float(p.A[b][0][0]) for b in range(2)]
        self.diff = [float(p.diffusivity[b][0][0]) for b in range(2)]
        self.R = c["R"][0][1].tolist()
        self.Rinv = c["Rinv"][0][1].tolist()
        self.R10 = c["R"][1][0].tolist()
        self.Rinv10 = c["Rinv"][1][0].tolist()
        self.ix = [_copy_map(self.mx, p.bc_type[f][0], p.bc_type[f][1]) for f in (0, 1)]
        self.iy = [_copy_map(self.my, p.bc_type[f][3], p.bc_type[f][2]) for f in (0, 1)]

    def theta0(self):
        p = self.p
        return torch.tensor([p.tau_ab[0][1], p.dab[0][1], p.epsilon, p.gamma[0][1]], dtype=torch.float64)

    # ---- helpers over the ghosted grid
    def ghost(self, f, a):
        """interior [mx][my] -> ghosted [rx][ry] by the boundary copy of field kind f"""
        return a[self.ix[f]][:, self.iy[f]]

    def h(self, pa):
        """hphi of a phase (functionH.h:24-36) for N = 2: no pair terms"""
        s = 3.0 * pa * pa - 2.0 * pa * pa * pa
        s1 = 0.0 * (2.0 * pa)
        return s + s1

    def cmu_of(self, m, b):
        return 0.0 + self.cmu[b] * (m - self.E[b])

    def dadq(self, q0, q1, dab):
        qx3, qy3 = q0 * q0 * q0, q1 * q1 * q1
        q2 = (q0 * q0 + q1 * q1) + 0.0 * 0.0
        ok = q2.abs() > 1.0e-15
        q2s = torch.where(ok, q2, torch.ones_like(q2))
        q22, q23 = q2s * q2s, q2s * q2s * q2s
        q4 = (qx3 * q0 + qy3 * q1) + 0.0 * 0.0 * 0.0 * 0.0
        d0 = 16.0 * dab * (qx3 / q22 - q0 * q4 / q23)
        d1 = 16.0 * dab * (qy3 / q22 - q1 * q4 / q23)
        z = torch.zeros_like(q0)
        return torch.where(ok, d0, z), torch.where(ok, d1, z)

    def ac(self, q0, q1, dab):
        qx2, qy2 = q0 * q0, q1 * q1
        qx4, qy4 = qx2 * qx2, qy2 * qy2
        q2 = (qx2 + qy2) + 0.0 * 0.0
        ok = q2.abs() > 1.0e-15
        q2s = torch.where(ok, q2, torch.ones_like(q2))
        v = 1.0 - dab * (3.0 - 4.0 * ((qx4 + qy4) + 0.0) / (q2s * q2s))
        return torch.where(ok, v, torch.ones_like(v))

    def step(self, phi, mu, theta):
        """phi [2][mx][my], mu [1][mx][my] -> the state after one step"""
        rx, ry, dx, dy, dt = self.rx, self.ry, self.dx, self.dy, self.dt
        tau01, dab, eps, gamma = theta[0], theta[1], theta[2], theta[3]
        P = [self.ghost(0, phi[a]) for a in range(2)]
        Mg = self.ghost(1, mu[0])

        # ---- phi faces (calculate_gradients.h:92-131) as windows: gx, sx over rows
        # [0, rx-1); gy, sy over columns [0, ry-1); gcy over columns [1, ry-1);
        # gcx over rows [1, rx-1)
        gx = [(p[1:, :] - p[:-1, :]) / dx for p in P]
        sx = [0.5 * (p[1:, :] + p[:-1, :]) for p in P]
        gy = [(p[:, 1:] - p[:, :-1]) / dy for p in P]
        sy = [0.5 * (p[:, 1:] + p[:, :-1]) for p in P]
        gcy = [(p[:, 2:] - p[:, :-2]) / (2.0 * dy) for p in P]
        gcx = [0.5 * (g[1:, :] + g[:-1, :]) for g in gx]

        # windows by absolute ghosted coordinates: rows [x0, x1), columns [y0, y1)
        def W(arr, ox, oy, x0, x1, y0, y1):
            return arr[x0 - ox:x1 - ox, y0 - oy:y1 - oy]

        # ---- delta-phi of the ring and interior: rows, columns [2, r-2)
        X0, X1, Y0, Y1 = 2, rx - 2, 2, ry - 2

        def fx(a, name, dxo=0, dyo=0):
            """face quantity of phase a at (x + dxo, y + dyo) over the delta-phi window"""
            arr, ox, oy = {"gx": (gx[a], 0, 0), "sx": (sx[a], 0, 0), "gy": (gy[a], 0, 0), "sy": (sy[a], 0, 0),
                           "gcy": (gcy[a], 0, 1), "gcx": (gcx[a], 1, 0)}[name]
            return W(arr, ox, oy, X0 + dxo, X1 + dxo, Y0 + dyo, Y1 + dyo)

        ph = [W(P[a], 0, 0, X0, X1, Y0, Y1) for a in range(2)]
        m = W(Mg, 0, 0, X0, X1, Y0, Y1)
        dv = [(fx(a, "gx") - fx(a, "gx", -1)) / dx + (fx(a, "gy") - fx(a, "gy", 0, -1)) / dy for a in range(2)]
        act = [d.abs() > 0.0 for d in dv]
        zero = torch.zeros_like(ph[0])

        def rot(a):
            return self.R if a == 0 else self.R10

        def rotinv(a):
            return self.Rinv if a == 0 else self.Rinv10

        def dA(a):
            b = 1 - a
            if not self.aniso:
                sp = 0.0 + (ph[a] * fx(b, "gcx") - ph[b] * fx(a, "gcx")) * fx(b, "gcx")
                sp = sp + (ph[a] * fx(b, "gcy") - ph[b] * fx(a, "gcy")) * fx(b, "gcy")
                sp = sp * gamma
                return 2.0 * (0.0 + sp)
            t0 = ph[a] * fx(b, "gcx") - ph[b] * fx(a, "gcx")
            t1 = ph[a] * fx(b, "gcy") - ph[b] * fx(a, "gcy")
            q0, q1 = _rot2(rot(a), t0, t1)
            d0, d1 = self.dadq(q0, q1, dab)
            q2 = (q0 * q0 + q1 * q1) + 0.0 * 0.0
            ac1 = self.ac(q0, q1, dab)
            ac2 = ac1 * ac1
            e0, e1 = _rot2(rot(a), fx(b, "gcx"), fx(b, "gcy"))
            sp1 = (0.0 + q0 * e0) + q1 * e1
            sp2 = (0.0 + d0 * e0) + d1 * e1
            sp1 = sp1 * (gamma * ac2)
            sp2 = sp2 * (gamma * ac1 * q2)
            return 2.0 * ((0.0 + sp1) + (0.0 + sp2))

        def qx_face(a, b, dxo):
            """q_divx at the face between x+dxo and x+dxo+1 (functionQ.h:4-21)"""
            t0 = fx(a, "sx", dxo) * fx(b, "gx", dxo) - fx(b, "sx", dxo) * fx(a, "gx", dxo)
            t1 = 0.5 * (fx(a, "sx", dxo) * (fx(b, "gcy", dxo) + fx(b, "gcy", dxo + 1)) -
                        fx(b, "sx", dxo) * (fx(a, "gcy", dxo) + fx(a, "gcy", dxo + 1)))
            return _rot2(rot(a), t0, t1)

        def qy_face(a, b, dyo):
            """q_divy at the face between y+dyo and y+dyo+1 (functionQ.h:22-40)"""
            t0 = 0.5 * (fx(a, "sy", 0, dyo) * (fx(b, "gcx", 0, dyo) + fx(b, "gcx", 0, dyo + 1)) -
                        fx(b, "sy", 0, dyo) * (fx(a, "gcx", 0, dyo) + fx(a, "gcx", 0, dyo + 1)))
            t1 = fx(a, "sy", 0, dyo) * fx(b, "gy", 0, dyo) - fx(b, "sy", 0, dyo) * fx(a, "gy", 0, dyo)
            return _rot2(rot(a), t0, t1)

        def divdA(a):
            b = 1 - a
            sxa, sxb, gxa, gxb = (lambda o: fx(a, "sx", o)), (lambda o: fx(b, "sx", o)), \
                (lambda o: fx(a, "gx", o)), (lambda o: fx(b, "gx", o))
            sya, syb, gya, gyb = (lambda o: fx(a, "sy", 0, o)), (lambda o: fx(b, "sy", 0, o)), \
                (lambda o: fx(a, "gy", 0, o)), (lambda o: fx(b, "gy", 0, o))
            if not self.aniso:
                d = ((sxa(0) * gxb(0) - sxb(0) * gxa(0)) * (-sxb(0)) -
                     ((sxa(-1) * gxb(-1) - sxb(-1) * gxa(-1)) * (-sxb(-1)))) / dx
                d = d + ((sya(0) * gyb(0) - syb(0) * gya(0)) * (-syb(0)) -
                         ((sya(-1) * gyb(-1) - syb(-1) * gya(-1)) * (-syb(-1)))) / dy
                d = d * gamma
                return 2.0 * (0.0 + d)
            qf, qb, qr, ql = qx_face(a, b, 0), qx_face(a, b, -1), qy_face(a, b, 0), qy_face(a, b, -1)
            acf, acb, acr, acl = (self.ac(q[0], q[1], dab) for q in (qf, qb, qr, ql))
            d1 = ((acf * acf * (sxa(0) * gxb(0) - sxb(0) * gxa(0)) * (-sxb(0))) -
                  (acb * acb * (sxa(-1) * gxb(-1) - sxb(-1) * gxa(-1)) * (-sxb(-1)))) / dx
            d1 = d1 + ((acr * acr * (sya(0) * gyb(0) - syb(0) * gya(0)) * (-syb(0))) -
                       (acl * acl * (sya(-1) * gyb(-1) - syb(-1) * gya(-1)) * (-syb(-1)))) / dy
            d1 = d1 * gamma

            def rd(q):
                d0, dd1 = self.dadq(q[0], q[1], dab)
                return _rot2(rotinv(a), d0, dd1), (q[0] * q[0] + q[1] * q[1]) + 0.0 * 0.0
            (rdf, qf2), (rdb, qb2), (rdr, qr2), (rdl, ql2) = rd(qf), rd(qb), rd(qr), rd(ql)
            d2 = (acf * qf2 * rdf[0] * (-sxb(0)) - acb * qb2 * rdb[0] * (-sxb(-1))) / dx
            d2 = d2 + (acr * qr2 * rdr[1] * (-syb(0)) - acl * ql2 * rdl[1] * (-syb(-1))) / dy
            d2 = d2 * gamma
            return 2.0 * ((0.0 + d1) + (0.0 + d2)) + 0.0

        def dwdphi(a):
            b = 1 - a
            if self.well:
                s = torch.where(act[b], 0.0 + 2.0 * gamma * (ph[b] * ph[b] * ph[a]), zero)
                return s * 9.0
            pos = (ph[a] * ph[b]) >= 0.0
            t = torch.where(pos, gamma * ph[b], -gamma * ph[b])
            s = torch.where(act[b], 0.0 + t, zero)
            return s * (16.0 / (math.pi * math.pi))

        def dpsi(a):
            s = zero
            for b in range(2):
                c = self.cmu_of(m, b)
                psi = 0.0 - m * c
                fe = ((0.0 + self.A[b] * c * c) + self.B[b] * c) + self.C[b]
                psi = psi + fe
                dh = 6.0 * ph[a] * (1.0 - ph[a]) if a == b else 0.0 * ph[b]
                s = s + psi * dh
            return s

        lam = [(eps * (-dA(a) + divdA(a)) - (1.0 / eps) * dwdphi(a)) - dpsi(a) for a in range(2)]
        sl, cnt = zero, torch.zeros_like(ph[0])
        for a in range(2):
            sl = torch.where(act[a], sl + lam[a], sl)
            cnt = cnt + act[a].to(torch.float64)
        sl = torch.where(cnt > 0, sl / torch.where(cnt > 0, cnt, torch.ones_like(cnt)), sl)
        s_t = 0.0 + tau01 * ph[0] * ph[1]
        s1_t = 0.0 + ph[0] * ph[1]
        nz = s1_t != 0.0
        tau = torch.where(nz, s_t / torch.where(nz, s1_t, torch.ones_like(s1_t)),
                          torch.full_like(s1_t, self.tau_default))
        d = [torch.where(act[a], dt * (lam[a] - sl) / (tau * eps), zero) for a in range(2)]
        d = self.project(ph, act, d)

        # ---- concentration pass over the interior
        I0, I1, J0, J1 = 3, rx - 3, 3, ry - 3

        def dphi_at(a, dxo=0, dyo=0, x0=I0, x1=I1, y0=J0, y1=J1):
            return W(d[a], X0, Y0, x0 + dxo, x1 + dxo, y0 + dyo, y1 + dyo)

        def Dcell(pa0, pa1):
            return (0.0 + self.diff[0] * self.cmu[0] * pa0) + self.diff[1] * self.cmu[1] * pa1

        def G(arr, x0, x1, y0, y1):
            return W(arr, 0, 0, x0, x1, y0, y1)

        def Dmx_gmx(x0, x1, y0, y1):
            """x-face flux D*grad mu between rows x and x+1"""
            Dm = (Dcell(G(P[0], x0 + 1, x1 + 1, y0, y1), G(P[1], x0 + 1, x1 + 1, y0, y1)) +
                  Dcell(G(P[0], x0, x1, y0, y1), G(P[1], x0, x1, y0, y1))) * 0.5
            gm = (G(Mg, x0 + 1, x1 + 1, y0, y1) - G(Mg, x0, x1, y0, y1)) / dx
            return Dm * gm

        def Dmy_gmy(x0, x1, y0, y1):
            Dm = (Dcell(G(P[0], x0, x1, y0 + 1, y1 + 1), G(P[1], x0, x1, y0 + 1, y1 + 1)) +
                  Dcell(G(P[0], x0, x1, y0, y1), G(P[1], x0, x1, y0, y1))) * 0.5
            gm = (G(Mg, x0, x1, y0 + 1, y1 + 1) - G(Mg, x0, x1, y0, y1)) / dy
            return Dm * gm

        divflux = 0.0 + (Dmx_gmx(I0, I1, J0, J1) - Dmx_gmx(I0 - 1, I1 - 1, J0, J1)) / dx
        divflux = divflux + (Dmy_gmy(I0, I1, J0, J1) - Dmy_gmy(I0, I1, J0 - 1, J1 - 1)) / dy

        L, a0 = 1, 0
        atf = 1.0 - self.diff[a0] / self.diff[L]

        def s_of(pa):
            """the obstacle anti-trapping weight of a cell"""
            w = pa * (1.0 - pa)
            ok = w > 0.0
            v = pa * (1.0 - self.h(pa)) / _Sqrt.apply(torch.where(ok, w, torch.ones_like(w)))
            return torch.where(ok, v, torch.zeros_like(v))

        def safe_sqrt(v):
            ok = v > 0.0
            return torch.where(ok, _Sqrt.apply(torch.where(ok, v, torch.ones_like(v))), torch.zeros_like(v))

        def jx(x0, x1, y0, y1):
            """anti-trapping current through the x-faces of rows [x0, x1)"""
            gxa = W(gx[a0], 0, 0, x0, x1, y0, y1)
            gxl = W(gx[L], 0, 0, x0, x1, y0, y1)
            gpy = 0.5 * (W(gcy[a0], 0, 1, x0, x1, y0, y1) + W(gcy[a0], 0, 1, x0 + 1, x1 + 1, y0, y1))
            ng = safe_sqrt(gpy * gpy + gxa * gxa)
            gpy_l = 0.5 * (W(gcy[L], 0, 1, x0, x1, y0, y1) + W(gcy[L], 0, 1, x0 + 1, x1 + 1, y0, y1))
            ngx_l = safe_sqrt(gpy_l * gpy_l + gxl * gxl)
            mc, mf = G(Mg, x0, x1, y0, y1), G(Mg, x0 + 1, x1 + 1, y0, y1)
            pc, pf = G(P[a0], x0, x1, y0, y1), G(P[a0], x0 + 1, x1 + 1, y0, y1)
            cl_f, cl_c = self.cmu_of(mf, L), self.cmu_of(mc, L)
            cs_f, cs_c = self.cmu_of(mf, a0), self.cmu_of(mc, a0)
            sp = gxa * gxl
            sp = sp + gpy * gpy_l
            okd = (ngx_l > 0.0) & (ng != 0.0)   # where ng is 0 the current is 0 whatever sp is
            sp = torch.where(ngx_l > 0.0, sp / torch.where(okd, ngx_l * ng, torch.ones_like(ng)), sp)
            dpf, dpc = dphi_at(a0, 1, 0, x0, x1, y0, y1), dphi_at(a0, 0, 0, x0, x1, y0, y1)
            ngs = torch.where(ng != 0.0, ng, torch.ones_like(ng))
            if self.well:
                t = atf * sp.abs() * (0.5 / math.sqrt(2.0)) * ((cl_f - cs_f) * dpf + (cl_c - cs_c) * dpc) * gxa / ngs
            else:
                t = atf * sp.abs() * 0.5 * (s_of(pf) * (cl_f - cs_f) * dpf + s_of(pc) * (cl_c - cs_c) * dpc) * gxa / ngs
            return torch.where(ng != 0.0, 0.0 + t, torch.zeros_like(t))

        def jy(x0, x1, y0, y1):
            """anti-trapping current through the y-faces of columns [y0, y1)"""
            gya = W(gy[a0], 0, 0, x0, x1, y0, y1)
            gyl = W(gy[L], 0, 0, x0, x1, y0, y1)
            gpx = 0.5 * (W(gcx[a0], 1, 0, x0, x1, y0, y1) + W(gcx[a0], 1, 0, x0, x1, y0 + 1, y1 + 1))
            ng = safe_sqrt(gpx * gpx + gya * gya)
            gpx_l = 0.5 * (W(gcx[L], 1, 0, x0, x1, y0, y1) + W(gcx[L], 1, 0, x0, x1, y0 + 1, y1 + 1))
            ngy_l = safe_sqrt(gpx_l * gpx_l + gyl * gyl)
            mc, mr = G(Mg, x0, x1, y0, y1), G(Mg, x0, x1, y0 + 1, y1 + 1)
            pc, pr = G(P[a0], x0, x1, y0, y1), G(P[a0], x0, x1, y0 + 1, y1 + 1)
            cl_r, cl_c = self.cmu_of(mr, L), self.cmu_of(mc, L)
            cs_r, cs_c = self.cmu_of(mr, a0), self.cmu_of(mc, a0)
            sp = gya * gyl
            sp = sp + gpx * gpx_l
            okd = (ngy_l > 0.0) & (ng != 0.0)
            sp = torch.where(ngy_l > 0.0, sp / torch.where(okd, ngy_l * ng, torch.ones_like(ng)), sp)
            dpr, dpc = dphi_at(a0, 0, 1, x0, x1, y0, y1), dphi_at(a0, 0, 0, x0, x1, y0, y1)
            ngs = torch.where(ng != 0.0, ng, torch.ones_like(ng))
            if self.well:
                t = atf * sp.abs() * (0.5 / math.sqrt(2.0)) * ((cl_r - cs_r) * dpr + (cl_c - cs_c) * dpc) * gya / ngs
            else:
                t = atf * sp.abs() * 0.5 * (s_of(pr) * (cl_r - cs_r) * dpr + s_of(pc) * (cl_c - cs_c) * dpc) * gya / ngs
            # the reference leaves the current of ghosted column MESH_Y - 2 at 0
            # (calculate_fluxes_concentration.h, the y != MESH_Y-2 guard)
            cols = torch.arange(y0, y1).unsqueeze(0)
            ok = (ng != 0.0) & (cols != 0) & (cols != self.my - 2)
            return torch.where(ok, 0.0 + t, torch.zeros_like(t))

        cst = (-0.25 * math.pi * eps) if not self.well else (-1.0 * eps)
        divjat = (jx(I0, I1, J0, J1) - jx(I0 - 1, I1 - 1, J0, J1)) * cst / dx
        divjat = divjat + (jy(I0, I1, J0, J1) - jy(I0, I1, J0 - 1, J1 - 1)) * cst / dy

        pi = [G(P[a], I0, I1, J0, J1) for a in range(2)]
        mi = G(Mg, I0, I1, J0, J1)
        di = [dphi_at(a) for a in range(2)]
        ssum = torch.zeros_like(mi)
        for a in range(2):
            sdh = 0.0
            for b in range(2):
                dh = 6.0 * pi[a] * (1.0 - pi[a]) if a == b else 0.0 * pi[a]
                sdh = sdh + dh * di[b]
            ssum = ssum + self.cmu_of(mi, a) * sdh
        # bulk cells: the first phase whose phi is exactly 1
        bulk0, bulk1 = pi[0] == 1.0, (pi[0] != 1.0) & (pi[1] == 1.0)
        nm_bulk = []
        for bph in range(2):
            cold = self.cmu_of(mi, bph)
            cnew = cold + dt * divflux - divjat
            nm_bulk.append(2.0 * self.A[bph] * cnew + self.E[bph])
        deltac = dt * divflux - divjat - ssum
        dcdmu = (0.0 + self.cmu[0] * self.h(pi[0])) + self.cmu[1] * self.h(pi[1])
        inter = ~(bulk0 | bulk1)
        dcs = torch.where(inter, dcdmu, torch.ones_like(dcdmu))
        nm_int = mi + deltac * (1.0 / dcs)
        nm = torch.where(bulk0, nm_bulk[0], torch.where(bulk1, nm_bulk[1], nm_int))
        nph = [pi[a] + di[a] for a in range(2)]
        return torch.stack(nph), nm.unsqueeze(0)

    def project(self, ph, act, d):
        """projection_on_simplex (simplex_projection.h:1-49) for two phases"""
        N = 2
        zero = torch.zeros_like(ph[0])
        d = list(d)
        inside = [act[a] & ((ph[a] + d[a]) > 0.0) & ((ph[a] + d[a]) < 1.0) for a in range(N)]
        count = sum(m.to(torch.float64) for m in inside)
        sum_phib = zero
        for a in range(N):
            sum_phib = torch.where(inside[a], sum_phib + ph[a], sum_phib)
        Dphi = zero
        for a in range(N):
            neg = (ph[a] + d[a]) < 0.0
            da = (d[a] + ph[a]).abs()
            d[a] = torch.where(neg, d[a] + da, d[a])
            Dphi = torch.where(neg, Dphi + da, Dphi)
        pos = Dphi > 0.0
        for b in range(N):
            mb = pos & act[b] & ((ph[b] + d[b]) > 0.0) & ((ph[b] + d[b]) < 1.0)
            nzs = sum_phib.abs() > 0.0
            w = torch.where(nzs, Dphi * ph[b] / torch.where(nzs, sum_phib, torch.ones_like(sum_phib)),
                            Dphi / torch.where(count > 0, count, torch.ones_like(count)))
            d[b] = torch.where(mb, d[b] - w, d[b])
        done = torch.zeros_like(act[0])
        for a in range(N):
            cond = (~done) & act[a] & ((ph[a] + d[a]) > 1.0)
            nd = list(d)
            nd[a] = torch.where(cond, 1.0 - ph[a], d[a])
            for b in range(N):
                if b != a:
                    nd[b] = torch.where(cond & act[b], -ph[b], d[b])
            d = nd
            done = done | cond
        return d

    def run(self, phi, mu, theta, nsteps):
        for _ in range(nsteps):
            phi, mu = self.step(phi, mu, theta)
        return phi, mu


def tape_gradients(p, phi0, mu0, nsteps, target=None, phi_bar=None):
    """Loss and gradients through nsteps tape steps: with target, L = 1/2
    sum (phi_T - target)^2; with phi_bar, L = sum phi_bar * phi_T.  Returns
    (loss, dL/dtheta [Tau, dab, epsilon, GAMMA], dL/dphi0, dL/dmu0)."""
    ts = TapeStep(p)
    th = ts.theta0().requires_grad_(True)
    a = torch.from_numpy(np.ascontiguousarray(phi0, dtype=np.float64)).requires_grad_(True)
    m = torch.from_numpy(np.ascontiguousarray(mu0, dtype=np.float64)).requires_grad_(True)
    ph, _ = ts.run(a, m, th, nsteps)
    if target is not None:
        loss = 0.5 * ((ph - torch.from_numpy(target)) ** 2).sum()
    else:
        loss = (torch.from_numpy(phi_bar) * ph).sum()
    loss.backward()
    return float(loss.detach()), th.grad.numpy(), a.grad.numpy(), m.grad.numpy()
