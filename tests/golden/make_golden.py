"""Golden fixtures for the oracle, from an independent transcription.

The reference (src/programs/pic2d.f90) cannot be built here and ships no
golden vectors. This script is a second, independent restatement of its step,
transcribed statement by statement from the Fortran into plain Python floats
(IEEE double, no fused operations) with the Fortran array bounds kept as index
offsets. It runs a tiny periodic case on one rank and writes the inputs and
the outputs of pusher, fieldsolver and countingsort to golden_step.npz.
tests/test_golden.py checks the C++ oracle against it.

Run:  python tests/golden/make_golden.py
"""
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


class F90:
    """Arrays with Fortran lower bounds: a[i, j] addresses element (i, j)."""

    def __init__(self, lo_i, hi_i, lo_j, hi_j, ncomp):
        self.lo_i, self.lo_j = lo_i, lo_j
        self.a = np.zeros((hi_i - lo_i + 1, hi_j - lo_j + 1, ncomp))

    def g(self, c, i, j):
        return float(self.a[i - self.lo_i, j - self.lo_j, c])

    def s(self, c, i, j, v):
        self.a[i - self.lo_i, j - self.lo_j, c] = v


# record components, pic2d.f90:52-67
EX, DEX_DY, EY, DEY_DX, EZ, DEZ_DX, DEZ_DY, DIVE, BX, DBX_DY, BY, DBY_DX, BZ, DBZ_DX, DBZ_DY, PAD1 = range(16)
GEX, GEY, GEZ, GPAD1, GBX, GBY, GBZ, GPAD2 = range(8)
JX, JY, JZ, RHO = range(4)


def sign1(b):
    """Fortran SIGN(1.0, b) for b != 0."""
    return 1.0 if b >= 0.0 else -1.0


class Step:
    def __init__(self, mx, my, dx, dy, dt, cva, mime, in0, compat):
        self.mx, self.my = mx, my
        self.dx, self.dy, self.dt, self.cva, self.mime, self.in0 = dx, dy, dt, cva, mime, in0
        self.idx, self.idy = 1.0 / dx, 1.0 / dy
        self.cva2 = cva * cva
        self.dth = dt / 2.0
        self.compat = compat
        self.emf = F90(0, mx + 1, 0, my + 1, 16)
        self.emfgrid = F90(0, mx + 1, 0, my + 1, 8)
        self.denjr = F90(0, mx + 2, 0, my + 2, 4)
        self.totene = [0.0, 0.0, 0.0, 0.0]

    # ---------------------------------------------------------- currentdeposit
    def currentdeposit(self, i1, i2, j1, j2, dx1, dx2, dy1, dy2, q0, uz):  # pic2d.f90:1226
        D = self.denjr
        qx = q0 * self.dx / self.dt
        qy = q0 * self.dy / self.dt
        im = (i1 + i2 + dx1 + dx2 + 1) * 0.5
        jm = (j1 + j2 + dy1 + dy2 + 1) * 0.5
        ir = min(min(i1, i2) + 1.0, max(max(i1, i2) + 0.0, im))
        jr = min(min(j1, j2) + 1.0, max(max(j1, j2) + 0.0, jm))
        fx1 = qx * (ir - i1 - dx1 - 0.5)
        fy1 = qy * (jr - j1 - dy1 - 0.5)
        fx2 = qx * (i2 + dx2 + 0.5 - ir)
        fy2 = qy * (j2 + dy2 + 0.5 - jr)
        wx1 = (ir - i1 + dx1 + 0.5) * 0.5
        wy1 = (jr - j1 + dy1 + 0.5) * 0.5
        wx2 = (ir - i2 + dx2 + 0.5) * 0.5
        wy2 = (jr - j2 + dy2 + 0.5) * 0.5
        D.s(JX, i1, j1, D.g(JX, i1, j1) + fx1 * (1.0 - wy1))
        D.s(JX, i1, j1 + 1, D.g(JX, i1, j1 + 1) + fx1 * wy1)
        D.s(JY, i1, j1, D.g(JY, i1, j1) + fy1 * (1.0 - wx1))
        D.s(JY, i1 + 1, j1, D.g(JY, i1 + 1, j1) + fy1 * wx1)
        D.s(JX, i2, j2, D.g(JX, i2, j2) + fx2 * (1.0 - wy2))
        D.s(JX, i2, j2 + 1, D.g(JX, i2, j2 + 1) + fx2 * wy2)
        D.s(JY, i2, j2, D.g(JY, i2, j2) + fy2 * (1.0 - wx2))
        D.s(JY, i2 + 1, j2, D.g(JY, i2 + 1, j2) + fy2 * wx2)
        dimid = im - i1 - 0.5
        djmid = jm - j1 - 0.5
        di = int(round(sign1(dimid)))
        dj = int(round(sign1(djmid)))
        dimid = abs(dimid)
        djmid = abs(djmid)
        s1 = dimid * djmid
        s2 = dimid - s1
        s3 = djmid - s1
        s4 = 1.0 - s1 - s2 - s3
        quz = q0 * uz
        D.s(JZ, i1, j1, D.g(JZ, i1, j1) + quz * s4)
        D.s(JZ, i1 + di, j1, D.g(JZ, i1 + di, j1) + quz * s2)
        D.s(JZ, i1, j1 + dj, D.g(JZ, i1, j1 + dj) + quz * s3)
        D.s(JZ, i1 + di, j1 + dj, D.g(JZ, i1 + di, j1 + dj) + quz * s1)
        if self.compat & 4:
            s1 = (0.5 - dx1) * (0.5 - dy1)
            s2 = 0.5 - dx1 - s1
            s3 = 0.5 - dy1 - s1
        else:  # the gather's weights
            s1 = (0.5 + dx1) * (0.5 + dy1)
            s2 = 0.5 + dx1 - s1
            s3 = 0.5 + dy1 - s1
        s4 = 1.0 - s1 - s2 - s3
        ix1, iy1 = i1 + 1, j1 + 1
        D.s(RHO, i1, j1, D.g(RHO, i1, j1) + s4 * q0)
        D.s(RHO, ix1, j1, D.g(RHO, ix1, j1) + s2 * q0)
        D.s(RHO, i1, iy1, D.g(RHO, i1, iy1) + s3 * q0)
        D.s(RHO, ix1, iy1, D.g(RHO, ix1, iy1) + s1 * q0)

    # ------------------------------------------------------------------ pusher
    def pusher(self, ptl):  # pic2d.f90:912-1217; ptl: list of dicts, modified in place
        mx, my = self.mx, self.my
        G = self.emfgrid
        nptltot = 10 ** 9
        sendt, sendb, crossindex = [], [], []
        ke = [0.0, 0.0]
        for i, p in enumerate(ptl):
            ux, uy, uz = p["ux"], p["uy"], p["uz"]
            ix = (p["grid"] - 1) // my + 1
            iy = (p["grid"] - 1) % my + 1
            s1 = (0.5 + p["dx"]) * (0.5 + p["dy"])
            s2 = 0.5 + p["dx"] - s1
            s3 = 0.5 + p["dy"] - s1
            s4 = 1.0 - s1 - s2 - s3

            def gat(c):
                return G.g(c, ix, iy) * s4 + G.g(c, ix + 1, iy) * s2 + G.g(c, ix, iy + 1) * s3 + \
                    G.g(c, ix + 1, iy + 1) * s1

            ex, ey, ez = gat(GEX), gat(GEY), gat(GEZ)
            bx, by, bz = gat(GBX), gat(GBY), gat(GBZ)
            ms = self.mime if p["q"] > 0 else 1.0
            c0 = p["q"] * self.dt * self.mime / ms / 2.0
            c1 = c0 / self.cva
            umx = ux + c1 * ex
            umy = uy + c1 * ey
            umz = uz + c1 * ez
            gama = math.sqrt(1.0 + umx * umx + umy * umy + umz * umz)
            c2 = c0 / gama
            tx, ty, tz = c2 * bx, c2 * by, c2 * bz
            t2 = 2.0 / (1.0 + tx * tx + ty * ty + tz * tz)
            sx, sy, sz = t2 * tx, t2 * ty, t2 * tz
            if self.compat & 1:
                vx, vy, vz_ = ux, uy, uz
            else:
                vx, vy, vz_ = umx, umy, umz
            u0x = umx + (vy * tz - vz_ * ty)
            u0y = umy + (vz_ * tx - vx * tz)
            u0z = umz + (vx * ty - vy * tx)
            upx = umx + (u0y * sz - u0z * sy)
            upy = umy + (u0z * sx - u0x * sz)
            upz = umz + (u0x * sy - u0y * sx)
            ux = upx + c1 * ex
            uy = upy + c1 * ey
            uz = upz + c1 * ez
            gama = math.sqrt(1.0 + ux * ux + uy * uy + uz * uz)
            p["ux"], p["uy"], p["uz"] = ux, uy, uz
            dx0, dy0 = p["dx"], p["dy"]
            c3 = self.dt * self.cva / gama
            dx1 = dx0 + c3 * ux * self.idx
            dy1 = dy0 + c3 * uy * self.idy
            if abs(dx1) > 0.5:
                dcellx = int(round(sign1(dx1)))
                p["dx"] = dx1 + sign1(-dx1)
            else:
                dcellx = 0
                p["dx"] = dx1
            if abs(dy1) > 0.5:
                dcelly = int(round(sign1(dy1)))
                p["dy"] = dy1 + sign1(-dy1)
            else:
                dcelly = 0
                p["dy"] = dy1
            ix1, iy1 = ix + dcellx, iy + dcelly
            vz = uz * self.cva / gama
            self.currentdeposit(ix, ix1, iy, iy1, dx0, p["dx"], dy0, p["dy"], p["q"], vz)
            ix = (ix1 + mx - 1) % mx + 1
            if iy1 > my:
                iy = iy1 - my
                p["grid"] = my * (ix - 1) + iy
                sendt.append(dict(p))
                p["pid"] = nptltot + 1
                crossindex.append(i)
            elif iy1 < 1:
                iy = iy1 + my
                p["grid"] = my * (ix - 1) + iy
                sendb.append(dict(p))
                p["pid"] = nptltot + 1
                crossindex.append(i)
            else:
                iy = iy1
                p["grid"] = my * (ix - 1) + iy
            j = 1 if p["q"] < 0 else 2
            ke[j - 1] += (gama - 1.0) * ms
        D = self.denjr
        D.a[:] = D.a * self.in0
        # compaction, pic2d.f90:1072-1083 (0-based positions)
        j = len(ptl) - 1
        for k in crossindex:
            while j >= 0 and ptl[j]["pid"] > nptltot:
                j -= 1
            if j < k:
                break
            ptl[k] = ptl[j]
            j -= 1
        del ptl[len(ptl) - len(crossindex):]
        ptl.extend(sendb)  # ptlrecvt: from the right neighbour (this rank)
        ptl.extend(sendt)  # ptlrecvb
        # x fold, pic2d.f90:1150-1169
        for jj in range(0, my + 3):
            for c in (JX, JY, JZ):
                D.s(c, 0, jj, D.g(c, 0, jj) + D.g(c, mx, jj))
                D.s(c, 1, jj, D.g(c, 1, jj) + D.g(c, mx + 1, jj))
                if c == JY and not (self.compat & 2):
                    D.s(c, 2, jj, D.g(c, 2, jj) + D.g(c, mx + 2, jj))
                D.s(c, mx, jj, D.g(c, 0, jj))
                D.s(c, mx + 1, jj, D.g(c, 1, jj))
                if c == JY and not (self.compat & 2):
                    D.s(c, mx + 2, jj, D.g(c, 2, jj))
            D.s(RHO, 1, jj, D.g(RHO, 1, jj) + D.g(RHO, mx + 1, jj))
            D.s(RHO, mx + 1, jj, D.g(RHO, 1, jj))
            D.s(RHO, 0, jj, D.g(RHO, mx, jj))
        # y guard exchange with itself, pic2d.f90:1171-1216
        sendt_ = [[D.g(JX, i, my + 1) for i in range(mx + 2)], [D.g(JX, i, my + 2) for i in range(mx + 2)],
                  [D.g(JY, i, my + 1) for i in range(mx + 2)], [D.g(JZ, i, my + 1) for i in range(mx + 2)],
                  [D.g(RHO, i, my + 1) for i in range(mx + 2)]]
        sendb_ = [[D.g(JX, i, 0) for i in range(mx + 2)], [D.g(JX, i, 1) for i in range(mx + 2)],
                  [D.g(JY, i, 0) for i in range(mx + 2)], [D.g(JZ, i, 0) for i in range(mx + 2)],
                  [D.g(RHO, i, 1) for i in range(mx + 2)]]
        recvb, recvt = sendt_, sendb_
        for i in range(mx + 2):
            D.s(JX, i, 1, D.g(JX, i, 1) + recvb[0][i])
            D.s(JX, i, 2, D.g(JX, i, 2) + recvb[1][i])
            D.s(JY, i, 1, D.g(JY, i, 1) + recvb[2][i])
            D.s(JZ, i, 1, D.g(JZ, i, 1) + recvb[3][i])
            D.s(RHO, i, 1, D.g(RHO, i, 1) + recvb[4][i])
            D.s(JX, i, my, D.g(JX, i, my) + recvt[0][i])
            D.s(JX, i, my + 1, D.g(JX, i, my + 1) + recvt[1][i])
            D.s(JY, i, my, D.g(JY, i, my) + recvt[2][i])
            D.s(JZ, i, my, D.g(JZ, i, my) + recvt[3][i])
            D.s(RHO, i, my + 1, D.g(RHO, i, my + 1) + recvt[4][i])
        self.totene[0], self.totene[1] = ke

    # ------------------------------------------------------------- fieldsolver
    def _periodic_x(self, comps):
        E, mx, my = self.emf, self.mx, self.my
        for c in comps:
            for j in range(my + 2):
                E.s(c, 0, j, E.g(c, mx, j))
                E.s(c, 1, j, E.g(c, mx + 1, j))

    def _exchange_y(self, ca, cb):
        E, mx, my = self.emf, self.mx, self.my
        top = [(E.g(ca, i, my), E.g(cb, i, my)) for i in range(mx + 2)]
        bot = [(E.g(ca, i, 1), E.g(cb, i, 1)) for i in range(mx + 2)]
        for i in range(mx + 2):
            E.s(ca, i, my + 1, bot[i][0])
            E.s(cb, i, my + 1, bot[i][1])
            E.s(ca, i, 0, top[i][0])
            E.s(cb, i, 0, top[i][1])

    def _b_half(self):
        E = self.emf
        for i in range(self.mx + 2):
            for j in range(self.my + 2):
                E.s(BX, i, j, E.g(BX, i, j) - self.dth * E.g(DEZ_DY, i, j))
                E.s(BY, i, j, E.g(BY, i, j) + self.dth * E.g(DEZ_DX, i, j))
                E.s(BZ, i, j, E.g(BZ, i, j) + self.dth * (E.g(DEX_DY, i, j) - E.g(DEY_DX, i, j)))

    def _curl_e(self):
        E, mx, my = self.emf, self.mx, self.my
        for j in range(1, my + 1):
            for i in range(mx + 2):
                E.s(DEX_DY, i, j, (E.g(EX, i, j + 1) - E.g(EX, i, j)) * self.idy)
        for j in range(my + 2):
            for i in range(0, mx + 1):
                E.s(DEY_DX, i, j, (E.g(EY, i + 1, j) - E.g(EY, i, j)) * self.idx)
            for i in range(1, mx + 2):
                E.s(DEZ_DX, i, j, (E.g(EZ, i, j) - E.g(EZ, i - 1, j)) * self.idx)
        for j in range(1, my + 2):
            for i in range(mx + 2):
                E.s(DEZ_DY, i, j, (E.g(EZ, i, j) - E.g(EZ, i, j - 1)) * self.idy)
        for j in range(my + 2):
            E.s(DEY_DX, mx + 1, j, E.g(DEY_DX, 1, j))

    def fieldsolver(self):  # pic2d.f90:678-860, one rank
        E, D, G, mx, my = self.emf, self.denjr, self.emfgrid, self.mx, self.my
        self._b_half()
        self._periodic_x((BX, BY, BZ))
        self._exchange_y(BY, BZ)
        for j in range(1, my + 1):
            for i in range(mx + 2):
                E.s(DBX_DY, i, j, (E.g(BX, i, j + 1) - E.g(BX, i, j)) * self.idy)
        for j in range(my + 2):
            for i in range(0, mx + 1):
                E.s(DBY_DX, i, j, (E.g(BY, i + 1, j) - E.g(BY, i, j)) * self.idx)
            for i in range(1, mx + 2):
                E.s(DBZ_DX, i, j, (E.g(BZ, i, j) - E.g(BZ, i - 1, j)) * self.idx)
        for j in range(1, my + 2):
            for i in range(mx + 2):
                E.s(DBZ_DY, i, j, (E.g(BZ, i, j) - E.g(BZ, i, j - 1)) * self.idy)
        for j in range(my + 2):
            E.s(DBY_DX, mx + 1, j, E.g(DBY_DX, 1, j))
        c = self.dt * self.cva2
        for i in range(mx + 2):
            for j in range(my + 2):
                E.s(EX, i, j, E.g(EX, i, j) + c * (E.g(DBZ_DY, i, j) - D.g(JX, i, j)))
                E.s(EY, i, j, E.g(EY, i, j) - c * (E.g(DBZ_DX, i, j) + D.g(JY, i, j)))
                E.s(EZ, i, j, E.g(EZ, i, j) + c * (E.g(DBY_DX, i, j) - E.g(DBX_DY, i, j) - D.g(JZ, i, j)))
        self._periodic_x((EX, EY, EZ))
        self._exchange_y(EY, EZ)
        self._curl_e()
        self._b_half()
        self._exchange_y(BY, BZ)
        for j in range(my + 2):
            for i in range(1, mx + 2):
                G.s(GEX, i, j, (E.g(EX, i, j) + E.g(EX, i - 1, j)) * 0.5)
                G.s(GBX, i, j, (E.g(BX, i, j) + E.g(BX, i - 1, j)) * 0.5)
        for j in range(1, my + 2):
            for i in range(mx + 2):
                G.s(GEY, i, j, (E.g(EY, i, j) + E.g(EY, i, j - 1)) * 0.5)
                G.s(GBY, i, j, (E.g(BY, i, j) + E.g(BY, i, j - 1)) * 0.5)
            for i in range(1, mx + 2):
                G.s(GEZ, i, j, (E.g(EZ, i, j) + E.g(EZ, i - 1, j) + E.g(EZ, i, j - 1) + E.g(EZ, i - 1, j - 1)) * 0.25)
                G.s(GBZ, i, j, (E.g(BZ, i, j) + E.g(BZ, i - 1, j) + E.g(BZ, i, j - 1) + E.g(BZ, i - 1, j - 1)) * 0.25)
        se = sb = 0.0
        for j in range(1, my + 1):
            for i in range(1, mx + 1):
                se += G.g(GEX, i, j) ** 2 + G.g(GEY, i, j) ** 2 + G.g(GEZ, i, j) ** 2
                sb += G.g(GBX, i, j) ** 2 + G.g(GBY, i, j) ** 2 + G.g(GBZ, i, j) ** 2
        self.totene[2] = 0.5 * se * self.mime / (self.cva2 * self.cva2 * self.in0)
        self.totene[3] = 0.5 * sb * self.mime / (self.cva2 * self.in0)

    def load_fields(self, yee6):
        """Primary fields from the canonical (6, mx, my+1) layout, guards and curl terms."""
        E, mx, my = self.emf, self.mx, self.my
        for c, comp in enumerate((EX, EY, EZ, BX, BY, BZ)):
            for i in range(mx):
                for j in range(my):
                    E.s(comp, i + 1, j + 1, float(yee6[c, i, j]))
            for j in range(1, my + 1):
                E.s(comp, 0, j, E.g(comp, mx, j))
                E.s(comp, mx + 1, j, E.g(comp, 1, j))
            for i in range(mx + 2):
                E.s(comp, i, 0, E.g(comp, i, my))
                E.s(comp, i, my + 1, E.g(comp, i, 1))
        self._curl_e()
        G = self.emfgrid
        for j in range(my + 2):
            for i in range(1, mx + 2):
                G.s(GEX, i, j, (E.g(EX, i, j) + E.g(EX, i - 1, j)) * 0.5)
                G.s(GBX, i, j, (E.g(BX, i, j) + E.g(BX, i - 1, j)) * 0.5)
        for j in range(1, my + 2):
            for i in range(mx + 2):
                G.s(GEY, i, j, (E.g(EY, i, j) + E.g(EY, i, j - 1)) * 0.5)
                G.s(GBY, i, j, (E.g(BY, i, j) + E.g(BY, i, j - 1)) * 0.5)
            for i in range(1, mx + 2):
                G.s(GEZ, i, j, (E.g(EZ, i, j) + E.g(EZ, i - 1, j) + E.g(EZ, i, j - 1) + E.g(EZ, i - 1, j - 1)) * 0.25)
                G.s(GBZ, i, j, (E.g(BZ, i, j) + E.g(BZ, i - 1, j) + E.g(BZ, i, j - 1) + E.g(BZ, i - 1, j - 1)) * 0.25)


def countingsort(ptl, mx, my):  # pic2d.f90:1303-1329
    ptlalloc = [0] * (mx * my)
    for p in ptl:
        ptlalloc[p["grid"] - 1] += 1
    counts = list(ptlalloc)
    k = 0
    for i in range(mx * my):
        j = ptlalloc[i]
        ptlalloc[i] = k
        k += j
    out = [None] * len(ptl)
    for p in ptl:
        j = p["grid"] - 1
        k = ptlalloc[j] + 1
        ptlalloc[j] = k
        out[k - 1] = p
    return out, counts


FIELDS = ("dx", "dy", "ux", "uy", "uz", "grid", "q", "pid")


def to_array(ptl):
    return np.array([tuple(p[f] for f in FIELDS) for p in ptl],
                    dtype=[(f, "<f8") for f in FIELDS[:5]] + [(f, "<i4") for f in FIELDS[5:]])


def make_case(seed, compat, mx=6, my=5, n=40):
    rng = np.random.default_rng(seed)
    params = dict(mx=mx, my=my, dx=0.05, dy=0.04, dt=0.0009, cva=15.0, mime=25.0, in0=1.0 / 291.0)
    ptl = []
    for k in range(n):
        ptl.append(dict(dx=float(rng.uniform(-0.5, 0.5)), dy=float(rng.uniform(-0.5, 0.5)),
                        ux=float(rng.normal(0, 0.3)), uy=float(rng.normal(0, 0.3)), uz=float(rng.normal(0, 0.3)),
                        grid=int(rng.integers(1, mx * my + 1)), q=int(1 if k % 2 == 0 else -1), pid=k + 1))
    yee = rng.normal(0, 0.05, (6, mx, my + 1))
    yee[5] += 1.0
    yee[:, :, my] = 0.0
    inputs = to_array(ptl)
    st = Step(compat=compat, **params)
    st.load_fields(yee)
    sorted_ptl, counts = countingsort(ptl, mx, my)
    sorted_ptl = [dict(p) for p in sorted_ptl]
    sorted_pid = np.array([p["pid"] for p in sorted_ptl], dtype=np.int32)
    st.pusher(sorted_ptl)
    j4 = np.array([[[st.denjr.g(c, i + 1, j + 1) for j in range(my + 1)] for i in range(mx)] for c in range(4)])
    ke = list(st.totene[:2])
    pushed = to_array(sorted_ptl)
    st.fieldsolver()
    comps = (EX, EY, EZ, BX, BY, BZ)
    f6 = np.array([[[st.emf.g(c, i + 1, j + 1) for j in range(my + 1)] for i in range(mx)] for c in comps])
    g8 = np.array([[[st.emfgrid.g(c, i + 1, j + 1) for c in range(8)] for j in range(my + 1)] for i in range(mx + 1)])
    return dict(params=np.array([mx, my, params["dx"], params["dy"], params["dt"], params["cva"], params["mime"],
                                 params["in0"], compat]),
                inputs=inputs, yee=yee, counts=np.array(counts, dtype=np.int32),
                sorted_pid=sorted_pid, pushed=pushed, j4=j4,
                fields=f6, emfgrid=g8, energies=np.array(ke + st.totene[2:]))


def main():
    out = {}
    for name, seed, compat in (("a", 11, 0), ("b", 12, 7)):
        case = make_case(seed, compat)
        for k, v in case.items():
            out[f"{name}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "golden_step.npz"), **out)
    print("wrote", os.path.join(HERE, "golden_step.npz"))


if __name__ == "__main__":
    main()
