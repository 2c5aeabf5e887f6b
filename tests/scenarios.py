"""Known-answer Riemann scenarios restated from the reference's own tests
(numerics/riemann_solver/hll_test.py and hllc_test.py): uniform field,
Mach-6 normal shocks in moving frames, quiescent gas, plug flow and a Mach-2.5
shock reflection. Each builder returns 1-D face states (neg, pos) and the
expected values the reference tests assert.
"""

import numpy as np

from oracle import swirlc_oracle as orc

GAMMA, R, CP, CV = orc.GAMMA, orc.R, orc.CP, orc.CV
DIMS = ('x', 'y', 'z')
VEL = ('u', 'v', 'w')


def normal_shock(m):
  """hll_test.py:76-86."""
  p1_p0 = (2.0 * GAMMA * m**2 - (GAMMA - 1.0)) / (GAMMA + 1.0)
  r1_r0 = (GAMMA + 1.0) * m**2 / ((GAMMA - 1.0) * m**2 + 2.0)
  return p1_p0, r1_r0, p1_p0 / r1_r0


def state(rho, vel, p, t):
  """Primitive + conservative face state from rho, (u,v,w), p, T."""
  u, v, w = vel
  ke = 0.5 * (u * u + v * v + w * w)
  e = CV * t + ke
  h = CP * t + ke
  prim = {'rho': rho, 'u': u, 'v': v, 'w': w, 'e': e, 'p': p, 'h': h}
  cons = {'rho': rho, 'rho_u': rho * u, 'rho_v': rho * v, 'rho_w': rho * w,
          'rho_e': rho * e}
  return prim, cons


def _vec(a, b, n, split):
  out = np.empty(n)
  out[:split] = a
  out[split:] = b
  return out


def two_states(s0, s1, n=16, split_neg=8, split_pos=7):
  """Face states with neg = s0 up to split_neg and pos = s0 up to split_pos:
  index 7 sees neg = s0, pos = s1 (the shock face of the reference tests)."""
  neg = {k: _vec(s0[k], s1[k], n, split_neg) for k in s0}
  pos = {k: _vec(s0[k], s1[k], n, split_pos) for k in s0}
  return neg, pos


def physical_flux(prim, dim):
  d = DIMS.index(dim)
  un = prim[VEL[d]]
  m = prim['rho'] * un
  f = {'rho': m, 'rho_u': m * prim['u'], 'rho_v': m * prim['v'],
       'rho_w': m * prim['w'], 'rho_e': m * prim['h']}
  f['rho_' + VEL[d]] = f['rho_' + VEL[d]] + prim['p']
  return f


def uniform(dim, n=16):
  """hll_test.py:94-152: s_l = u_n - c, s_r = u_n + c (HLLC s_m = u_n)."""
  t, p = 500.0, 101325.0
  rho = p / (R * t)
  prim, cons = state(rho * np.ones(n), (10.0 * np.ones(n), 20.0 * np.ones(n),
                                         -5.0 * np.ones(n)), p * np.ones(n),
                     t * np.ones(n))
  c = np.sqrt(GAMMA * R * t)
  un = prim[VEL[DIMS.index(dim)]]
  return dict(neg=prim, pos=prim, cneg=cons, cpos=cons, s_l=un - c,
              s_r=un + c, s_m=un)


def _shock_pair(dim, m, frame, order, sign=1.0):
  """Pre/post states of a normal shock of Mach m (upstream speed sign*u0),
  plus the frame velocity, ordered (neg, pos) by `order`."""
  t0, p0 = 300.0, 101325.0
  u0 = sign * m * np.sqrt(GAMMA * R * t0)
  if callable(frame):
    frame = frame(u0)
  p1_p0, r1_r0, t1_t0 = normal_shock(m)
  fac = np.array([1.0, 1.0 / r1_r0])[order]
  pr = np.array([1.0, p1_p0])[order] * p0
  tt = np.array([1.0, t1_t0])[order] * t0
  vel = [250.0 * np.ones(2), 100.0 * np.ones(2), -200.0 * np.ones(2)]
  vel[DIMS.index(dim)] = fac * u0 + frame
  rho = pr / (R * tt)
  return rho, vel, pr, tt, u0


def shock_speeds(dim, left_running=True, n=16):
  """hll_test.py:154-338: uniform sides across a Mach-6 normal shock seen in
  a frame moving at -500. Left-running (u0 > 0, neg = pre-shock): s_l is the
  shock speed -500 and s_r = u~ + c~; right-running (u0 < 0, neg =
  post-shock): s_l = u~ - c~ and s_r = -500. Velocities are (shock, 100,
  -200) rotated so the shock velocity lies along `dim`."""
  m, t0, p0, frame = 6.0, 300.0, 101325.0, -500.0
  sign = 1.0 if left_running else -1.0
  u0 = sign * m * np.sqrt(GAMMA * R * t0)
  p1_p0, r1_r0, t1_t0 = normal_shock(m)
  order = [0, 1] if left_running else [1, 0]
  un = np.array([1.0, 1.0 / r1_r0])[order] * u0 + frame
  p = np.array([1.0, p1_p0])[order] * p0
  t = np.array([1.0, t1_t0])[order] * t0
  rho = p / (R * t)
  tv = [100.0 * np.ones(2), -200.0 * np.ones(2)]
  d = DIMS.index(dim)
  # (u, v, w) with the shock velocity along dim; the others keep 100/-200
  # in the reference's rotation (x: (un, 100, -200), y: (100, un, -200),
  # z: (-200, 100, un)).
  if d == 0:
    vel = [un, tv[0], tv[1]]
  elif d == 1:
    vel = [tv[0], un, tv[1]]
  else:
    vel = [tv[1], tv[0], un]
  h = CP * t + 0.5 * (vel[0]**2 + vel[1]**2 + vel[2]**2)
  rs = np.sqrt(rho)
  ravg = lambda f: np.sum(rs * f) / np.sum(rs)
  ru = [ravg(vel[0]), ravg(vel[1]), ravg(vel[2])]
  rh = ravg(h)
  roe_c = np.sqrt(GAMMA * R * (rh - 0.5 * (ru[0]**2 + ru[1]**2 + ru[2]**2))
                  / CP)
  s0 = state(rho[0] * np.ones(n), [v[0] * np.ones(n) for v in vel],
             p[0] * np.ones(n), t[0] * np.ones(n))[0]
  s1 = state(rho[1] * np.ones(n), [v[1] * np.ones(n) for v in vel],
             p[1] * np.ones(n), t[1] * np.ones(n))[0]
  if left_running:
    s_l, s_r = frame * np.ones(n), (roe_c + ru[d]) * np.ones(n)
  else:
    s_l, s_r = (ru[d] - roe_c) * np.ones(n), frame * np.ones(n)
  return dict(neg=s0, pos=s1, s_l=s_l, s_r=s_r)


def quiescent(dim, n=16):
  """hll_test.py:457-555: flux is p on the aligned momentum only."""
  t, p = 300.0, 101325.0
  rho = p / (R * t)
  z = np.zeros(n)
  prim, cons = state(rho * np.ones(n), (z, z, z), p * np.ones(n),
                     t * np.ones(n))
  exp = {k: np.zeros(n) for k in orc.BASE_CONSERVATIVE}
  exp['rho_' + VEL[DIMS.index(dim)]] = p * np.ones(n)
  return dict(neg=prim, pos=prim, cneg=cons, cpos=cons, flux=exp)


def plug(dim, n=16):
  """hll_test.py:557-668: identical sides; flux = physical flux."""
  p = 101325.0 * np.ones(n)
  t = np.linspace(300.0, 3000.0, n)
  rho = p / (R * t)
  prim, cons = state(rho, (10.0 * np.ones(n), -15.0 * np.ones(n),
                           25.0 * np.ones(n)), p, t)
  return dict(neg=prim, pos=prim, cneg=cons, cpos=cons,
              flux=physical_flux(prim, dim))


def uniform_pair(dim, m, frame, order, sign=1.0, n=16):
  rho, vel, pr, tt, u0 = _shock_pair(dim, m, frame, order, sign)
  s0, c0 = state(rho[0] * np.ones(n), [v[0] * np.ones(n) for v in vel],
                 pr[0] * np.ones(n), tt[0] * np.ones(n))
  s1, c1 = state(rho[1] * np.ones(n), [v[1] * np.ones(n) for v in vel],
                 pr[1] * np.ones(n), tt[1] * np.ones(n))
  return s0, c0, s1, c1, u0


def s_l_positive(dim):
  """hll_test.py:670-790: left-running Mach-6 shock in a crossflow of
  +0.5 u0, so s_r > s_l > 0 and the flux is F_neg."""
  s0, c0, s1, c1, _ = uniform_pair(dim, 6.0, lambda u0: 0.5 * u0, [0, 1])
  return dict(neg=s0, pos=s1, cneg=c0, cpos=c1, flux=physical_flux(s0, dim))


def s_r_negative(dim):
  """hll_test.py:794-926: right-running Mach-6 shock (u0 < 0) in a crossflow
  of 0.5 u0, so s_l < s_r < 0 and the flux is F_pos."""
  s0, c0, s1, c1, _ = uniform_pair(dim, 6.0, lambda u0: 0.5 * u0, [1, 0],
                                   sign=-1.0)
  return dict(neg=s0, pos=s1, cneg=c0, cpos=c1, flux=physical_flux(s1, dim))


def star_region(dim):
  """hll_test.py:928-1057: left-running Mach-6 shock, frame -0.4 u0; the
  right wave is acoustic and the flux equals F_pos."""
  s0, c0, s1, c1, _ = uniform_pair(dim, 6.0, lambda u0: -0.4 * u0, [0, 1])
  return dict(neg=s0, pos=s1, cneg=c0, cpos=c1, flux=physical_flux(s1, dim))


def shock_reflection(dim, n=16):
  """hll_test.py:1059-1228: two Mach-2.5 shocks meeting; only the aligned
  momentum flux is non-zero: rho u^2 + p + rho u s with s the Roe c."""
  m, t0, p0 = 2.5, 300.0, 101325.0
  u0 = m * np.sqrt(GAMMA * R * t0)
  p1_p0, r1_r0, t1_t0 = normal_shock(m)
  u1_u0 = 1.0 / r1_r0
  d = DIMS.index(dim)
  vel = [250.0 * np.ones(2), 100.0 * np.ones(2), -200.0 * np.ones(2)]
  vel[d] = np.array([1.0, -1.0]) * (1.0 - u1_u0) * u0
  p = np.ones(2) * p1_p0 * p0
  t = np.ones(2) * t1_t0 * t0
  rho = p / (R * t)
  s0, c0 = state(rho[0] * np.ones(n), [v[0] * np.ones(n) for v in vel],
                 p[0] * np.ones(n), t[0] * np.ones(n))
  s1, c1 = state(rho[1] * np.ones(n), [v[1] * np.ones(n) for v in vel],
                 p[1] * np.ones(n), t[1] * np.ones(n))
  vc = vel[d][0]
  roe_h = CP * t[0] + 0.5 * vc**2
  s = np.sqrt(GAMMA * R * roe_h / CP)
  exp = {k: np.zeros(n) for k in orc.BASE_CONSERVATIVE}
  exp['rho_' + VEL[d]] = (rho[0] * vc**2 + p[0] + rho[0] * vc * s) * np.ones(n)
  return dict(neg=s0, pos=s1, cneg=c0, cpos=c1, flux=exp)


FLUX_CASES = {
    'quiescent': quiescent, 'plug': plug, 's_l_positive': s_l_positive,
    's_r_negative': s_r_negative, 'star_region': star_region,
    'shock_reflection': shock_reflection,
}
