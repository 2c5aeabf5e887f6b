"""GPU: the discrete adjoint of whole runs (swc_rk_stage_vjp through
swirlc_b200.adjoint) against float64 central differences of the same runs,
h = 1e-6 (1e-8 for MUSCL) along seeded random directions in (initial
state, nu), for WENO5 and MUSCL (each limiter) with HLLC and HLL; plus the
autograd front end.

The scheme is only piecewise differentiable: HLLC sets s_m to 0 where
|s_m| < 1e-6 (hllc.py:328-341) and the wave-speed estimates take min / max
of two candidates that nearly tie in smooth flow (hll.py:265-283). Central
differences straddling such a kink differ from the derivative of the branch
taken (which is what the adjoint, like GradientTape, returns). The strict
bar (1e-6) is therefore checked on rough random states, where candidates
are well separated and s_m is generically far from 0; the smooth
Kelvin-Helmholtz set-up keeps the prescribed 16-direction check with a 1e-3
bar."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

NAMES = ('rho', 'rho_u', 'rho_v', 'rho_w', 'rho_e')


def _setup(user_cfg, state, dtype=torch.float64, nu=None):
  from swirlc_b200 import engine
  from swirlc_b200.core import parameter
  from swirlc_b200.physics import physics_models
  cfg = parameter.SwirlCParameters(user_cfg)
  f = [torch.tensor(state[k], dtype=dtype, device='cuda') for k in NAMES]
  s = engine.Solver(cfg, physics_models.PhysicsModels(cfg), f[0].shape, dtype)
  if nu is not None:
    s.scheme.nu = nu
  return cfg, s, f


def _loss(s, fields):
  from swirlc_b200 import adjoint
  return adjoint.vorticity_energy(fields, s.hw, s.grid.dx, s.grid.dy,
                                  s.grid.dz)


def _linear_loss(weights):
  """Seeded linear functional of the final state, balanced per field."""
  def loss(s, fields):
    return sum((w * f).sum() for w, f in zip(weights, fields))
  return loss


def _loss_grad(s, fields, loss=_loss):
  x = [f.detach().clone().requires_grad_(True) for f in fields]
  j = loss(s, x)
  g = torch.autograd.grad(j, x, allow_unused=True)
  return [torch.zeros_like(f) if gi is None else gi for f, gi in zip(fields, g)]


def _check_fd(user_cfg, state, steps, k, dts, ndir, seed=0, tol=1e-6,
              with_nu=True, linear=False, h=1e-6):
  from swirlc_b200 import adjoint
  cfg, s, f = _setup(user_cfg, state)
  loss = _loss
  if linear:
    rng_w = np.random.default_rng(100 + seed)
    hw = s.hw
    ws = []
    for x in f:
      w = torch.zeros_like(x)
      inner_ = (slice(hw, -hw),) * 3
      scale = float(x[inner_].abs().max()) or 1.0
      w[inner_] = torch.tensor(rng_w.standard_normal(x[inner_].shape) / scale,
                               dtype=x.dtype, device='cuda')
      ws.append(w)
    loss = _linear_loss(ws)
  nu0 = float(s.scheme.nu)
  run = adjoint.RunAdjoint(s, checkpoint_every=k)
  out = run.run(f, dts)
  grad, nub = run.backward(_loss_grad(s, out, loss))
  hw = s.hw
  inner = (slice(hw, -hw),) * 3
  rng = np.random.default_rng(seed)
  worst = 0.0
  for _ in range(ndir):
    d = []
    for x in f:
      scale = float(x[inner].abs().max()) or 1.0
      dd = torch.zeros_like(x)
      dd[inner] = torch.tensor(rng.standard_normal(x[inner].shape) * scale,
                               dtype=x.dtype, device='cuda')
      d.append(dd)
    dnu = float(rng.standard_normal()) * nu0 if with_nu else 0.0
    js = []
    for sgn in (1.0, -1.0):
      s.scheme.nu = nu0 + sgn * h * dnu
      r2 = adjoint.RunAdjoint(s, checkpoint_every=k)
      o2 = r2.run([x + sgn * h * dx for x, dx in zip(f, d)], dts)
      js.append(float(loss(s, o2)))
    s.scheme.nu = nu0
    fd = (js[0] - js[1]) / (2 * h)
    ad = sum(float((g[inner] * dx[inner]).sum()) for g, dx in zip(grad, d))
    ad += nub * dnu
    rel = abs(fd - ad) / max(abs(fd), abs(ad), 1e-30)
    worst = max(worst, rel)
    assert rel <= tol, (fd, ad, rel)
  return worst


def _rough(state, seed, p_scale=1.0, pe=None):
  """Random state of the same shape: rho in [1, 2], u in [-1, 1]^3,
  p in p_scale * [1, 2] (plus the potential energy rho * pe)."""
  rng = np.random.default_rng(seed)
  shape = state['rho'].shape
  rho = rng.uniform(1.0, 2.0, shape)
  u = rng.uniform(-1.0, 1.0, (3,) + shape)
  p = p_scale * rng.uniform(1.0, 2.0, shape)
  e_pot = 0.0 if pe is None else rho * pe
  return {'rho': rho, 'rho_u': rho * u[0], 'rho_v': rho * u[1],
          'rho_w': rho * u[2],
          'rho_e': p / 0.4 + 0.5 * rho * (u ** 2).sum(0) + e_pot}


def test_rough_periodic_viscous_gradient_matches_fd():
  from swirlc_b200 import configs
  cfg, state = configs.kelvin_helmholtz(n=8, nu=1e-2, dtype=np.float64)
  _check_fd(cfg, _rough(state, 7), 4, 2, [1e-3] * 4, ndir=16, seed=0)


def test_rough_inviscid_neumann_walls_gradient_matches_fd():
  from swirlc_b200 import configs
  cfg, state = configs.sod(n=16, ny=6, nz=6, dtype=np.float64)
  _check_fd(cfg, _rough(state, 8), 3, 2, [5e-4] * 3, ndir=8, seed=1,
            with_nu=False, linear=True)


def test_rough_gravity_dirichlet_walls_gradient_matches_fd():
  from oracle import swirlc_oracle as orc
  from swirlc_b200 import configs
  cfg, state = configs.buoyant_bubble(nx=6, ny=6, nz=10, dtype=np.float64)
  cfg = dict(cfg, interpolation_scheme='WENO_5', numeric_flux_scheme='HLLC',
             include_diffusion=True,
             transport_parameters={'nu': 1e-1, 'pr': 0.7})
  keys = ('halo_width', 'dx', 'dy', 'dz', 'x', 'y', 'z', 'g',
          'source_functions')
  ocfg = orc.make_cfg(**{k: cfg[k] for k in keys if k in cfg})
  pe = orc.potential_energy(ocfg, state['rho'].shape, np.float64)
  st = _rough(state, 9, p_scale=1e5, pe=pe)
  _check_fd(cfg, st, 3, 2, [1e-5] * 3, ndir=8, seed=2, linear=True)


@pytest.mark.parametrize('interp,riemann,limiter', [
    ('WENO_5', 'HLL', 'mc'),
    ('MUSCL', 'HLLC', 'van_leer'),
    ('MUSCL', 'HLL', 'van_leer'),
    ('MUSCL', 'HLL', 'mc'),
    ('MUSCL', 'HLL', 'minmod'),
    ('MUSCL', 'HLL', 'minmod3'),
])
def test_rough_scheme_variants_gradient_matches_fd(interp, riemann, limiter):
  """HLL and the MUSCL limiters on the rough periodic viscous case. The
  limiters switch branch where dm / dp crosses 0, 1/3, 1 or 3, and on a
  rough state many slopes lie near a switch: at h = 1e-6 a direction
  straddles one now and then (minmod: up to 1.3e-4 measured), at h = 1e-7
  rarely, at h = 1e-8 never in these directions (all <= 1.2e-7, float64
  rounding; 1e-9 typical where nothing is straddled). Hence h = 1e-8."""
  from swirlc_b200 import configs
  cfg, state = configs.kelvin_helmholtz(n=8, nu=1e-2, dtype=np.float64)
  cfg = dict(cfg, interpolation_scheme=interp, numeric_flux_scheme=riemann,
             muscl_limiter=limiter)
  _check_fd(cfg, _rough(state, 11), 3, 2, [1e-3] * 3, ndir=8, seed=3,
            h=1e-8)


def test_muscl_hll_gravity_walls_gradient_matches_fd():
  """The buoyant bubble's scheme (MUSCL van Leer + HLL, gravity,
  Dirichlet / Neumann z walls) on a rough state."""
  from oracle import swirlc_oracle as orc
  from swirlc_b200 import configs
  cfg, state = configs.buoyant_bubble(nx=6, ny=6, nz=10, dtype=np.float64)
  keys = ('halo_width', 'dx', 'dy', 'dz', 'x', 'y', 'z', 'g',
          'source_functions')
  ocfg = orc.make_cfg(**{k: cfg[k] for k in keys if k in cfg})
  pe = orc.potential_energy(ocfg, state['rho'].shape, np.float64)
  st = _rough(state, 12, p_scale=1e5, pe=pe)
  _check_fd(cfg, st, 3, 2, [1e-5] * 3, ndir=8, seed=4, with_nu=False,
            linear=True, h=1e-8)


def test_kh_benchmark_setup_gradient_matches_fd():
  """The adjoint benchmark's set-up (KH, viscous, vorticity energy) with
  the prescribed 16 directions; 1e-3 because the smooth flow crosses the
  scheme's kinks (module docstring)."""
  from swirlc_b200 import configs
  cfg, state = configs.kelvin_helmholtz(n=12, nu=1e-2, dtype=np.float64)
  _check_fd(cfg, state, 7, 3, [2e-3] * 7, ndir=16, seed=0, tol=1e-3)


def test_autograd_front_end_matches_reverse_sweep():
  from swirlc_b200 import adjoint, configs
  cfg, state = configs.kelvin_helmholtz(n=12, nu=1e-2, dtype=np.float64)
  _, s, f = _setup(cfg, state)
  dts = [2e-3] * 4
  run = adjoint.RunAdjoint(s, checkpoint_every=2)
  x = [t.clone().requires_grad_(True) for t in f]
  nu = torch.tensor(float(s.scheme.nu), dtype=torch.float64,
                    requires_grad=True)
  out = adjoint.simulate(run, x, dts, nu)
  loss = _loss(s, out)
  loss.backward()
  run2 = adjoint.RunAdjoint(s, checkpoint_every=4)
  o2 = run2.run(f, dts)
  g2, nub2 = run2.backward(_loss_grad(s, o2))
  hw = s.hw
  inner = (slice(hw, -hw),) * 3
  for a, b in zip(x, g2):
    torch.testing.assert_close(a.grad[inner], b[inner], rtol=1e-12, atol=0)
  assert float(nu.grad) == pytest.approx(nub2, rel=1e-12)


def test_second_simulate_on_one_runner_is_refused_at_backward():
  """A runner keeps the checkpoints of its latest run: the backward of an
  earlier simulate() after a second one raises instead of reversing the
  later trajectory; the later graph's backward still works and restores its
  own nu."""
  from swirlc_b200 import adjoint, configs
  cfg, state = configs.kelvin_helmholtz(n=12, nu=1e-2, dtype=np.float64)
  _, s, f = _setup(cfg, state)
  run = adjoint.RunAdjoint(s, checkpoint_every=2)
  nu1 = torch.tensor(1e-2, dtype=torch.float64, requires_grad=True)
  nu2 = torch.tensor(3e-2, dtype=torch.float64, requires_grad=True)
  x = [t.clone().requires_grad_(True) for t in f]
  out1 = adjoint.simulate(run, x, [2e-3] * 3, nu1)
  out2 = adjoint.simulate(run, x, [2e-3] * 3, nu2)
  with pytest.raises(RuntimeError, match='run again'):
    _loss(s, out1).backward()
  s.scheme.nu = 0.5  # changed by the caller in between
  _loss(s, out2).backward()
  assert s.scheme.nu == pytest.approx(3e-2)
  ref = adjoint.RunAdjoint(s, checkpoint_every=2)
  s.scheme.nu = 3e-2
  o = ref.run(f, [2e-3] * 3)
  _, nub = ref.backward(_loss_grad(s, o))
  assert float(nu2.grad) == pytest.approx(nub, rel=1e-9)


def test_stored_stages_match_checkpointed_sweep():
  """checkpoint_every=0 keeps every stage state instead of recomputing: the
  recomputed stage states are the forward run's bit for bit, and every sum
  of the stage adjoint has a fixed order, so the gradient is the same to
  the bit."""
  from swirlc_b200 import adjoint, configs
  cfg, state = configs.kelvin_helmholtz(n=12, nu=1e-2, dtype=np.float64)
  _, s, f = _setup(cfg, state)
  dts = [2e-3] * 5
  res = []
  for k in (0, 2):
    run = adjoint.RunAdjoint(s, checkpoint_every=k)
    o = run.run(f, dts)
    res.append(run.backward(_loss_grad(s, o)))
  for a, b in zip(res[0][0], res[1][0]):
    assert torch.equal(a, b)
  assert res[0][1] == res[1][1]


def test_backward_twice_gives_the_same_gradient():
  from swirlc_b200 import adjoint, configs
  cfg, state = configs.kelvin_helmholtz(n=12, nu=1e-2, dtype=np.float64)
  _, s, f = _setup(cfg, state)
  run = adjoint.RunAdjoint(s, checkpoint_every=2, steps=5)
  o = run.run(f, [2e-3] * 5)
  g = _loss_grad(s, o)
  a, na = run.backward(g)
  b, nb = run.backward(g)
  for x, y in zip(a, b):
    assert torch.equal(x, y)
  assert na == nb


@pytest.mark.parametrize('case', ['kh_viscous', 'bubble_walls'])
def test_gradients_are_bit_reproducible(case):
  """Two independent runners on the same float32 inputs give the same
  gradient bits: no sum of the stage adjoint depends on the order in which
  threads finish. Lines of 40 cells span three face segments per thread
  line (heads shared by two threads), the viscous case moves tangential
  cotangents onto neighbouring lines, and the walls case gathers the halo
  cotangents of Neumann and Dirichlet sides."""
  from oracle import swirlc_oracle as orc
  from swirlc_b200 import adjoint, configs
  if case == 'kh_viscous':
    cfg, state = configs.kelvin_helmholtz(n=40, nu=1e-3, dtype=np.float64)
    dts = [1e-3] * 4
  else:
    cfg, state = configs.buoyant_bubble(nx=20, ny=18, nz=40,
                                        dtype=np.float64)
    keys = ('halo_width', 'dx', 'dy', 'dz', 'x', 'y', 'z', 'g',
            'source_functions')
    ocfg = orc.make_cfg(**{k: cfg[k] for k in keys if k in cfg})
    pe = orc.potential_energy(ocfg, state['rho'].shape, np.float64)
    state = _rough(state, 13, p_scale=1e5, pe=pe)
    dts = [1e-2] * 4
  res = []
  for _ in range(2):
    _, s, f = _setup(cfg, state, torch.float32)
    run = adjoint.RunAdjoint(s, checkpoint_every=2)
    o = run.run(f, dts)
    res.append(run.backward(_loss_grad(s, o)))
  for a, b in zip(res[0][0], res[1][0]):
    assert torch.isfinite(a).all()
    assert torch.equal(a, b)
  assert res[0][1] == res[1][1]


def test_float32_adjoint_agrees_with_float64():
  from swirlc_b200 import adjoint, configs
  cfg, state = configs.kelvin_helmholtz(n=16, nu=1e-2, dtype=np.float64)
  dts = [2e-3] * 4
  grads = {}
  for dt_ in (torch.float32, torch.float64):
    _, s, f = _setup(cfg, state, dt_)
    run = adjoint.RunAdjoint(s, checkpoint_every=2)
    o = run.run(f, dts)
    g, nub = run.backward(_loss_grad(s, o))
    grads[dt_] = ([x.double() for x in g], nub)
  hw = 3
  inner = (slice(hw, -hw),) * 3
  # Whole gradient within 1e-3, each field within 1e-2 (float32 rounding,
  # and branch choices at the scheme's kinks can differ between precisions).
  num = den = 0.0
  for a, b in zip(grads[torch.float32][0], grads[torch.float64][0]):
    da = float((a[inner] - b[inner]).norm())
    db = float(b[inner].norm())
    assert da <= 1e-2 * db, (da, db)
    num += da * da
    den += db * db
  assert (num / den) ** 0.5 <= 1e-3
  assert grads[torch.float32][1] == pytest.approx(grads[torch.float64][1],
                                                  rel=1e-3)


def test_adjoint_rejects_unsupported_schemes():
  from swirlc_b200 import adjoint, configs
  cfg, state = configs.sod(n=24, ny=4, nz=4, dtype=np.float64)
  cfg = dict(cfg, interpolation_scheme='WENO_3')
  _, s, f = _setup(cfg, state)
  run = adjoint.RunAdjoint(s, checkpoint_every=2)
  o = run.run(f, [1e-3])
  with pytest.raises(NotImplementedError):
    run.backward(_loss_grad(s, o))


@pytest.mark.parametrize('scheme', ['rk3', 'rk2'])
def test_step_vjp_equals_its_stage_vjps(scheme):
  """swc_rk_step_vjp (one call per reversed step) gives the bits of its two
  or three swc_rk_stage_vjp calls made one by one."""
  from swirlc_b200 import adjoint, configs
  cfg, state = configs.kelvin_helmholtz(n=16, nu=1e-2, dtype=np.float64)
  _, s, f = _setup(cfg, state, torch.float32)
  run = adjoint.RunAdjoint(s, checkpoint_every=0, scheme=scheme)
  run.run(f, [2e-3] * 2)
  stages = run._pool[1]
  gen = torch.Generator(device='cuda').manual_seed(5)
  g = [torch.randn(x.shape, generator=gen, device='cuda') for x in f]
  outs = []
  for fn in (run._reverse_step, run._reverse_step_by_stage):
    run._nu_bar.zero_()
    gn, g2, g1 = (s.new_fields(zero=True) for _ in range(3))
    fn(stages, 2e-3, g, gn, g2, g1)
    outs.append(([x.clone() for x in gn], float(run._nu_bar.item())))
  for a, b in zip(outs[0][0], outs[1][0]):
    assert torch.equal(a, b)
  assert outs[0][1] == outs[1][1] != 0.0
