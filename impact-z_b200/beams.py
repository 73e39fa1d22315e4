"""Seeded synthetic bunches and lattices of the benchmark configurations.

Bunches are written in the reference's particle.in / Pts1 layout
(readin_Dist, src/Appl/Distribution.f90:1666-1714): 9 columns per particle
x/Scxl, gamma*beta_x, y/Scxl, gamma*beta_y, phase[rad], gamma0-gamma, q/m,
charge weight, id, with the charge weight Current/Scfreq/Npt*sign(q)
(Distribution.f90:245).  Random numbers come from numpy's Philox counter-based
generator (4x64, 10 rounds) keyed by the seed, so every run of a
configuration sees the same particles.
"""
import math

import numpy as np

CLIGHT = 299792458.0
PROTON_MASS_EV = 938.27208816e6
ELECTRON_MASS_EV = 0.51099895000e6
SEED0 = 20261203


def scxl(freq):
    """PhysConst Scxl = c/(2 pi f) (src/DataStruct/PhysConst.f90:30)."""
    return CLIGHT / (2 * (2 * math.asin(1.0)) * freq)


def _truncated_normal(rng, shape, trunc):
    z = rng.standard_normal(shape)
    if trunc is not None:
        bad = np.abs(z) > trunc
        while bad.any():
            z[bad] = rng.standard_normal(int(bad.sum()))
            bad = np.abs(z) > trunc
    return z


def refptcl_for(ekin, mass, phase=0.0):
    """construct_BeamBunch's refptcl (BeamBunch.f90:56-58)."""
    r = np.zeros(6)
    r[4] = phase
    r[5] = -(ekin / mass + 1.0)
    return r


def gaussian_bunch(n, seed=SEED0, mass=PROTON_MASS_EV, charge=1.0, ekin=2.5e6, current=0.030,
                   freq=402.5e6, sig_x=1e-3, sig_y=1e-3, sig_xp=1e-3, sig_yp=1e-3,
                   sig_phase_deg=5.0, sig_e=50e3, trunc=4.0):
    """Uncorrelated 6D Gaussian truncated at `trunc` sigma per coordinate.

    sig_x/y in m, sig_xp/yp in rad, phase in degrees, energy spread in eV."""
    rng = np.random.Generator(np.random.Philox(key=seed))
    z = _truncated_normal(rng, (6, n), trunc)
    gam0 = 1.0 + ekin / mass
    gb0 = math.sqrt(gam0 * gam0 - 1.0)
    xl = scxl(freq)
    pts = np.empty((n, 9))
    pts[:, 0] = z[0] * (sig_x / xl)
    pts[:, 1] = z[1] * (sig_xp * gb0)
    pts[:, 2] = z[2] * (sig_y / xl)
    pts[:, 3] = z[3] * (sig_yp * gb0)
    pts[:, 4] = z[4] * math.radians(sig_phase_deg)
    pts[:, 5] = z[5] * (sig_e / mass)
    pts[:, 6] = charge / mass
    pts[:, 7] = current / freq / n * charge / abs(charge)
    pts[:, 8] = np.arange(1, n + 1, dtype=np.float64)
    return pts, refptcl_for(ekin, mass)


AMU_EV = 931.49410242e6


def charge_state_bunch(nptlist, charge_states, currlist, seed=SEED0, mass_number=238,
                       ekin_per_u=0.5e6, freq=80.5e6, **kw):
    """An ion bunch of several charge states (Distribution.f90:1360-1367):
    charge state j holds nptlist[j] particles with Pts1(7) = Q_j / mass and
    Pts1(8) = currlist[j] / freq / nptlist[j] (signed like Q_j), interleaved
    at random; the coordinates are one truncated 6D Gaussian (gaussian_bunch's
    keywords).  The reference particle has the first charge state.  Returns
    (pts, refptcl, mass, qmcclist)."""
    mass = mass_number * AMU_EV
    n = int(sum(nptlist))
    pts, ref = gaussian_bunch(n, seed=seed, mass=mass, charge=charge_states[0],
                              ekin=ekin_per_u * mass_number, current=1.0, freq=freq, **kw)
    rng = np.random.Generator(np.random.Philox(key=seed + 1))
    state = rng.permutation(np.repeat(np.arange(len(nptlist)), nptlist))
    qmc = np.array([q / mass for q in charge_states])
    w = np.array([c / freq / m * math.copysign(1.0, q)
                  for c, m, q in zip(currlist, nptlist, charge_states)])
    pts[:, 6] = qmc[state]
    pts[:, 7] = w[state]
    return pts, ref, mass, qmc


def flat_top_bunch(n, seed=SEED0, mass=ELECTRON_MASS_EV, charge=-1.0, ekin=250e6 - ELECTRON_MASS_EV,
                   current=100.0, freq=1.3e9, length=1e-3, mod_amp=0.01, mod_lambda=10e-6,
                   sig_x=0.2e-3, sig_xp=0.02e-3, sig_e=5e3, trunc=4.0):
    """Flat-top longitudinal profile with a sinusoidal density modulation
    (rejection sampled), Gaussian transverse, uncorrelated energy spread."""
    rng = np.random.Generator(np.random.Philox(key=seed))
    gam0 = 1.0 + ekin / mass
    gb0 = math.sqrt(gam0 * gam0 - 1.0)
    beta0 = gb0 / gam0
    xl = scxl(freq)
    zpos = np.empty(0)
    while zpos.size < n:
        m = int((n - zpos.size) * 1.1) + 1024
        cand = rng.uniform(-length / 2, length / 2, m)
        keep = rng.uniform(0, 1 + mod_amp, m) < 1 + mod_amp * np.cos(2 * np.pi * cand / mod_lambda)
        zpos = np.concatenate([zpos, cand[keep]])
    zpos = zpos[:n]
    t = _truncated_normal(rng, (5, n), trunc)
    pts = np.empty((n, 9))
    pts[:, 0] = t[0] * (sig_x / xl)
    pts[:, 1] = t[1] * (sig_xp * gb0)
    pts[:, 2] = t[2] * (sig_x / xl)
    pts[:, 3] = t[3] * (sig_xp * gb0)
    # phase = -omega*z/(beta c) in the reference's units (z>0 is the head)
    pts[:, 4] = -zpos / (beta0 * xl)
    pts[:, 5] = t[4] * (sig_e / mass)
    pts[:, 6] = charge / mass
    pts[:, 7] = current / freq / n * charge / abs(charge)
    pts[:, 8] = np.arange(1, n + 1, dtype=np.float64)
    return pts, refptcl_for(ekin, mass)


def fodo(periods=10, gradient=20.0, ldrift=0.1, lquad=0.1, nseg=4, mapstp=1, radius=1.0):
    """[drift, quad(+G), drift, quad(-G)] x periods; quads in gradient mode
    (file ID 0, Quadrupole.f90:19-28)."""
    from . import elem
    out = []
    for _ in range(periods):
        out.append(elem(0, ldrift, nseg, mapstp, [radius]))
        out.append(elem(1, lquad, nseg, mapstp, [gradient, 0.0, radius]))
        out.append(elem(0, ldrift, nseg, mapstp, [radius]))
        out.append(elem(1, lquad, nseg, mapstp, [-gradient, 0.0, radius]))
    return out


def chicane(angle_deg=3.0, lbend=0.2, ldrift_in=20.0, ldrift_mid=3.5, ldrift_c=0.5, nseg_bend=8,
            nseg_drift=4, drift_steps_in=756, half_gap=0.01, file_id=150.0):
    """20 m of drift then a 4-dipole chicane (+a, -a, -a, +a sector bends);
    800 steps by default.  R56 = -2 a^2 (ldrift_mid + 2 lbend / 3) is about
    -20 mm for 3 degree bends 3.5 m apart.
    Dipole deck values: v1 angle[rad], v2 k1, v3 file ID (150: z map + SC,
    no CSR; above 200: CSR inside the bends; above 500: also the transient
    CSR downstream), v4 half gap (Dipole.f90:19-31,
    AccSimulator.f90:1035-1074, 1131-1138)."""
    from . import elem
    a = math.radians(angle_deg)

    def bend(sgn):
        return elem(4, lbend, nseg_bend, 1, [sgn * a, 0.0, file_id, half_gap, 0.0, 0.0, 0.0, 0.0,
                                             0.0])

    out = [elem(0, ldrift_in, drift_steps_in, 1, [1.0])]
    out += [bend(+1), elem(0, ldrift_mid, nseg_drift, 1, [1.0]), bend(-1),
            elem(0, ldrift_c, nseg_drift, 1, [1.0]), bend(-1),
            elem(0, ldrift_mid, nseg_drift, 1, [1.0]), bend(+1)]
    return out


# benchmark configurations -------------------------------------------------
def fodo_1e5(n=100_000, seed=SEED0):
    """Proton FODO, 1e5 particles, 32x32x64, 160 steps (plain FP64)."""
    pts, ref = gaussian_bunch(n, seed)
    return dict(pts=pts, refptcl=ref, current=0.030, mass=PROTON_MASS_EV, charge=1.0,
                freq=402.5e6, grid=(32, 32, 64), lattice=fodo(10))


def fodo_4e6(n=4_000_000, seed=SEED0, periods=25, nseg=10):
    """The same beam with 4e6 particles on 64x64x128; 25 FODO periods with
    10 steps per element = 1000 steps."""
    pts, ref = gaussian_bunch(n, seed)
    return dict(pts=pts, refptcl=ref, current=0.030, mass=PROTON_MASS_EV, charge=1.0,
                freq=402.5e6, grid=(64, 64, 128), lattice=fodo(periods, nseg=nseg))


def fodo_steps(nsteps, gradient=20.0, ldrift=0.1, lquad=0.1, nseg=10, radius=1.0):
    """The 4e6-particle FODO pattern (10 steps per 0.1 m element) cut to exactly
    `nsteps` space-charge steps; a final partial element keeps the step length."""
    from . import elem
    pattern = [(0, ldrift, [radius]), (1, lquad, [gradient, 0.0, radius]),
               (0, ldrift, [radius]), (1, lquad, [-gradient, 0.0, radius])]
    out, left, i = [], int(nsteps), 0
    while left > 0:
        t, length, vals = pattern[i % 4]
        k = min(nseg, left)
        out.append(elem(t, length * k / nseg, k, 1, vals))
        left -= k
        i += 1
    return out


def scan_jobs(nbunch=256, seed=SEED0, nmin=1e4, nmax=2e6, steps_periods=25):
    """A batched parameter scan: independent proton bunches built as in fodo_1e5 with
    particle counts log-uniform in [nmin, nmax], grids drawn from {16^3,
    32x32x64, 64x64x128}, quad gradient U[10,20] T/m, current U[5,50] mA,
    25 FODO periods of 4 steps per element (400 steps).  Gradients stop at
    20 T/m: for 2.5 MeV protons the 0.1 m quadrupole / 0.1 m drift cell is
    unstable above about 22 T/m (focal length below half the half-cell),
    the beam grows without bound and the exact drift's square root turns
    negative.  Returns dicts with the lattice and the bunch's seed."""
    rng = np.random.Generator(np.random.Philox(key=seed + 7777))
    grids = [(16, 16, 16), (32, 32, 64), (64, 64, 128)]
    out = []
    for i in range(nbunch):
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        grid = grids[int(rng.integers(0, 3))]
        grad = float(rng.uniform(10.0, 20.0))
        cur = float(rng.uniform(0.005, 0.050))
        out.append(dict(index=i, n=n, grid=grid, gradient=grad, current=cur,
                        lattice=fodo(steps_periods, gradient=grad), seed=seed + 1000 + i))
    return out


def make_scan_bunch(job):
    pts, ref = gaussian_bunch(job["n"], seed=job["seed"], current=job["current"])
    return pts, ref


def serve_jobs(njobs, rate, seed=SEED0, nmin=1e4, nmax=4e6, smax=2000):
    """A served job stream: a Poisson stream of proton jobs (arrival rate `rate`/s),
    particle counts log-uniform in [nmin, nmax], grid from {32^3, 64^3,
    64x64x128}, 10-50 FODO periods with gradient U[10,20] T/m (the stable
    range, see scan_jobs), and 100-2000 steps (the period count is cut to the
    drawn step count)."""
    rng = np.random.Generator(np.random.Philox(key=seed + 9999))
    grids = [(32, 32, 32), (64, 64, 64), (64, 64, 128)]
    t = 0.0
    out = []
    for i in range(njobs):
        t += float(rng.exponential(1.0 / rate))
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        grid = grids[int(rng.integers(0, 3))]
        periods = int(rng.integers(10, 51))
        grad = float(rng.uniform(10.0, 20.0))
        steps = min(int(rng.integers(100, min(smax, 2000) + 1)), periods * 16)
        lat = fodo_steps(steps, gradient=grad, nseg=4)
        out.append(dict(index=i, arrival=t, n=n, grid=grid, gradient=grad, steps=steps,
                        lattice=lat, seed=seed + 5000 + i))
    return out
