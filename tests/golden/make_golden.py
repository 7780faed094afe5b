"""Generate the golden fixtures in tests/golden/ from the reference implementation.

Run where the reference sources are available, with $HELIUM_REFERENCE naming the
reference checkout (the folder that holds its python/ directory):

    make -C oracle && HELIUM_REFERENCE=<reference checkout> python tests/golden/make_golden.py

The reference's Python imports its native Fortran library at import time
(python/native.py:8).  No Fortran compiler exists here, so the library slot is
filled with this repository's C restatement (oracle/_build/libhelium_oracle.so,
itself pinned to the reference's independent Kronecker assembly).  Every golden
H·psi below is taken from reference code that does NOT go through that library:
``Helium.reference_sparse`` (python/helium3d.py:105-123, Kronecker assembly) and
``TorchHamiltonian`` (python/torch_backend.py:11-138, PyTorch complex128 on CPU).
Arnoldi, CF4/GMRES, flux and Volkov goldens also come from the reference's own
torch/numpy code.  The fixtures are small (tiny grids, seeded inputs) and are
committed; the GPU box never needs the reference.
"""
import json
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
if 'HELIUM_REFERENCE' not in os.environ:
    sys.exit('set HELIUM_REFERENCE to the reference checkout (the folder holding python/)')
REFERENCE = Path(os.environ['HELIUM_REFERENCE'])
os.environ['HELIUM_LIBRARY'] = str(REPO / 'oracle' / '_build' / 'libhelium_oracle.so')
os.environ.setdefault('OMP_NUM_THREADS', '4')
sys.path.insert(0, str(REFERENCE / 'python'))

import torch  # noqa: E402
from fedvr import make_grid  # noqa: E402
from helium3d import Helium  # noqa: E402
from coupled_angular import CoupledHelium  # noqa: E402
from torch_backend import TorchHamiltonian, exponential_action as torch_expaction  # noqa: E402
from propagate import exponential_action as cpu_expaction  # noqa: E402
from implicit import SeparablePreconditioner, cf4_step, gmres  # noqa: E402
from pulses import Pulse  # noqa: E402

torch.set_num_threads(4)


def tables(h):
    """Every array the device operator consumes, as stored by the reference."""
    out = {}
    for name in ('ptr', 'col', 'tv', 'diag', 'vptr', 'vc', 'vl', 'vcoef', 'rad', 'dptr', 'dc', 'de', 'dcoef', 'ldiff',
                 'r', 'exchange'):
        out['t_' + name] = np.asarray(getattr(h, name))
    return out


def save(name, **arrays):
    path = HERE / f'{name}.npz'
    np.savez_compressed(path, **arrays)
    print(f'{path.name}: {path.stat().st_size / 1024:.1f} KiB')


GRID_CASES = {
    'plain': dict(edges=[0, .5, 1, 2, 4], order=3),
    'ecs': dict(edges=[0, .5, 1, 2, 4], order=3, ecs_angle=.3, tail=5),
    'ecs_cut': dict(edges=[0, .5, 1, 2, 4, 6, 8], order=3, ecs_angle=.4, tail=8),
    'bridge': dict(edges=[0, 1, 2, 4, 8], order=6, ecs_angle=.5, tail=20),
    'variable': dict(edges=[0, 1, 2, 3], order=(3, 4, 5), ecs_angle=.3, tail=4, alpha=.8),
    'long_tail': dict(edges=[0, .5, 1, 2, 4, 8, 16, 20], order=6, ecs_angle=.5, tail=40, alpha=.8),
}


def grids():
    arrays = {'cases': json.dumps(GRID_CASES)}
    for key, args in GRID_CASES.items():
        g = make_grid(**args)
        arrays[f'{key}_r'] = g.r
        arrays[f'{key}_weights'] = g.weights
        arrays[f'{key}_kinetic'] = g.kinetic.toarray()
        arrays[f'{key}_interior'] = g.interior_weights
    save('grids', **arrays)


def apply_goldens(h, x, field, op):
    out = {}
    for velocity in (False, True):
        key = 'velocity' if velocity else 'length'
        out[f'kron_{key}'] = h.reference_sparse(field, velocity) @ x
        out[f'torch_{key}'] = op.host(op.apply(op.state(x), field, velocity))
    return out


def product_cases():
    # python tests/test_kernels.py:31-37 grid and field (Kronecker vs kernel).
    h = Helium(make_grid(**GRID_CASES['ecs']), 1, M=None)
    rng = np.random.default_rng(49)
    x = rng.normal(size=h.size) + 1j * rng.normal(size=h.size)
    f = np.array([.13, .23, .34])
    op = TorchHamiltonian(h, 'cpu')
    save('apply_ecs', x=x, field=f, shape=np.array(h.shape), lmax=1, M=-99, **tables(h),
         diag_parts=np.array(0), **apply_goldens(h, x, f, op))

    # python tests/test_torch_backend.py:8-20 (cutoff, surface, Arnoldi).
    g = make_grid(**GRID_CASES['ecs_cut'])
    h = Helium(g, 1, M=None, cutoff_radii=[1, 2])
    idx = h.prepare_surface(5)
    rng = np.random.default_rng(386)
    x = rng.normal(size=h.size) + 1j * rng.normal(size=h.size)
    x /= np.linalg.norm(x)
    f = np.array([.13, .23, .34])
    op = TorchHamiltonian(h, 'cpu', coulomb_backend='blocks')
    gold = apply_goldens(h, x, f, op)
    flux = h.flux(x, f)
    flux_torch = op.flux(op.state(x), f)
    y, info = torch_expaction(lambda v: op.apply(v, f), op.state(x), .02, tol=1e-11)
    z, zinfo = cpu_expaction(lambda v: op.host(op.apply(op.state(v), f, True)), x, .02, tol=1e-11)
    save('apply_cut', x=x, field=f, shape=np.array(h.shape), lmax=1, M=-99, cutoff=np.array([1., 2.]),
         surface_radius=5.0, surface_indices=idx, surface_T=h.surface_T, surface_P=h.surface_P,
         flux=flux, flux_torch=flux_torch, arnoldi_torch=op.host(y), arnoldi_torch_dim=info['dimension'],
         arnoldi_cpu=z, arnoldi_cpu_dim=zinfo['dimension'], arnoldi_dt=.02, arnoldi_tol=1e-11,
         **tables(h), **gold)


def coupled_case():
    # python tests/test_coupled_angular.py:6-17.
    u = Helium(make_grid([0, .5, 1, 2, 4, 6, 8], 3, ecs_angle=.4, tail=6), 2, M=0, cutoff_radii=[1, 2])
    c = CoupledHelium(u, 2)
    idx = c.prepare_surface(5)
    rng = np.random.default_rng(619)
    x = rng.normal(size=c.size) + 1j * rng.normal(size=c.size)
    f = np.array([0., 0., .15])
    op = TorchHamiltonian(c, 'cpu')
    gold = apply_goldens(c, x, f, op)
    save('apply_coupled', x=x, field=f, shape=np.array(c.shape), lmax=2, total_Lmax=2, cutoff=np.array([1., 2.]),
         grid=json.dumps(dict(edges=[0, .5, 1, 2, 4, 6, 8], order=3, ecs_angle=.4, tail=6)),
         transform=c.transform, exchange_sign=c.exchange_sign, surface_indices=idx, flux=c.flux(x, f),
         **tables(c), **gold)


def bipolar_case():
    # Bipolar all-M basis (python/bipolar.py): the reference's own tables, and H·psi from two
    # paths that do not use the native library: the Kronecker assembly of the product basis
    # projected by the bipolar isometry (U^T H_product U x), and TorchHamiltonian on the
    # bipolar tables.  Field with all three Cartesian components (circular/elliptic probes).
    from bipolar import BipolarHelium
    args = dict(edges=[0, .5, 1, 2, 4, 6, 8], order=3, ecs_angle=.4, tail=6)
    g = make_grid(**args)
    b = BipolarHelium(g, lmax=2, total_Lmax=2, M=None, cutoff_radii=[1, 2])
    product = Helium(g, 2, M=None, cutoff_radii=[1, 2])
    U = b.transform.toarray()
    n2 = b.n * b.n
    rng = np.random.default_rng(733)
    x = rng.normal(size=b.size) + 1j * rng.normal(size=b.size)
    f = np.array([.11, -.07, .15])
    op = TorchHamiltonian(b, 'cpu')
    gold = {}
    for velocity in (False, True):
        key = 'velocity' if velocity else 'length'
        up = (x.reshape(n2, b.nc, order='F') @ U.T).ravel(order='F')
        hp = product.reference_sparse(f, velocity) @ up
        gold[f'kron_{key}'] = (hp.reshape(n2, product.nc, order='F') @ U).ravel(order='F')
        gold[f'torch_{key}'] = op.host(op.apply(op.state(x), f, velocity))
    save('apply_bipolar', x=x, field=f, shape=np.array(b.shape), lmax=2, total_Lmax=2, cutoff=np.array([1., 2.]),
         grid=json.dumps(args), basis=np.array(b.basis, np.int32), transform=U, exchange_sign=b.exchange_sign,
         product_channels=np.array([[a[0], a[1], c[0], c[1]] for a, c in product.ch], np.int32),
         **tables(b), **gold)


def ionic_adjoint_case():
    # Backward CF4-Pade propagation of the dual He+ channel functions with the ionic
    # Hamiltonian's adjoint (python/streaming_surface.py:125-146 with sparse LU,
    # python/implicit.py:111-123), velocity gauge, from t = 1.8 back to 1.0 in steps of 0.02.
    from surface3d import Ionic
    from streaming_surface import AdjointStepper
    args = dict(edges=[0, 1, 2, 3, 4, 6, 8, 10, 12], order=4, ecs_angle=.3, tail=8)
    base = Helium(make_grid(**args), 1, M=0, cutoff_radii=[3, 4])
    ion = Ionic(base, {0})
    unique = [(1, 0, 0), (2, 0, 0), (2, 1, 0)]
    pulse = Pulse(omega=2.0, cycles=2, field=.3)
    avec = lambda t: np.array([0., 0., float(pulse.vector(t))])
    stepper = AdjointStepper(ion, avec, 'cf4', 'lu')
    chi = ion.dual_final_states(unique)
    stepper.reset(chi)
    dt, t_end, steps = .02, 1.8, 40
    states = [chi]
    for i in range(steps):
        states.append(stepper.step(t_end - i * dt, -dt).copy())
    save('ionic_adjoint', grid=json.dumps(args), cutoff=np.array([3., 4.]), unique=np.array(unique),
         pulse=json.dumps(dict(omega=2.0, cycles=2, field=.3)), dt=dt, t_end=t_end, states=np.array(states))


def mixed_gauge_case():
    # Mixed length/velocity gauge operator (python/mixed_gauge.py:73-117) on CPU torch: the
    # coupled M = 0 case with a z field and the bipolar all-M case with a general field;
    # field = (A, E, six quadratic coefficients A_a A_b) as python/mixed_gauge.py:30-33 forms it.
    from mixed_gauge import MixedHamiltonian, parameters
    from bipolar import BipolarHelium
    out = {}
    args = dict(edges=[0, .5, 1, 2, 4, 6, 8], order=3, ecs_angle=.4, tail=6)
    g = make_grid(**args)
    cases = {'coupled': (CoupledHelium(Helium(g, 2, M=0, cutoff_radii=[1, 2]), 2), lambda t: np.array([0, 0, .21]),
                         lambda t: np.array([0, 0, -.13])),
             'bipolar': (BipolarHelium(g, lmax=1, total_Lmax=2, M=None, cutoff_radii=[1, 2]),
                         lambda t: np.array([.11, -.07, .15]), lambda t: np.array([-.05, .09, .04]))}
    for key, (h, avec, efunc) in cases.items():
        op = MixedHamiltonian(h, 'cpu', inner=1.5, outer=3.5)
        rng = np.random.default_rng(811)
        x = rng.normal(size=h.size) + 1j * rng.normal(size=h.size)
        field = parameters(avec, efunc, 0.)
        out[f'{key}_x'] = x
        out[f'{key}_field'] = field
        out[f'{key}_y'] = op.host(op.apply(op.state(x), field))
        out[f'{key}_y0'] = op.host(op.apply(op.state(x), np.zeros(12)))
    save('mixed_gauge', grid=json.dumps(args), cutoff=np.array([1., 2.]), inner=1.5, outer=3.5, **out)


def bipolar_contraction_case():
    # Ionic contraction of a surface frame in the bipolar all-M basis (sparse angular
    # transform, unfolded labels): python/surface_contract.py:29-37 and 49-56.
    from bipolar import BipolarHelium
    from surface3d import Ionic
    from surface_contract import SurfaceContractor as RefContractor
    args = dict(edges=[0, 1, 2, 3, 4, 6, 8, 10, 12], order=4, ecs_angle=.3, tail=8)
    h = BipolarHelium(make_grid(**args), lmax=1, total_Lmax=1, M=None, cutoff_radii=[3, 4])
    base = h.uncoupled
    idx = base.prepare_surface(8.)
    ion = Ionic(base, None)
    labels = [(1, 0, 0), (2, 0, 0), (2, 1, -1), (2, 1, 0), (2, 1, 1)]
    contract = RefContractor(base, ion, labels, labels, list(range(len(labels))), False, h.transform)
    rng = np.random.default_rng(97)
    chi = rng.normal(size=(ion.na * h.n, len(labels))) + 1j * rng.normal(size=(ion.na * h.n, len(labels)))
    frame = rng.normal(size=(h.n, len(idx), h.nc)) + 1j * rng.normal(size=(h.n, len(idx), h.nc))
    save('bipolar_contraction', grid=json.dumps(args), cutoff=np.array([3., 4.]), surface=8., labels=np.array(labels),
         chi=chi, frame=frame, q=contract(chi, frame), outer=np.array(contract.outerstates))


def arnoldi_dense():
    # python tests/test_kernels.py:42-47.
    from scipy.linalg import expm
    rng = np.random.default_rng(762)
    A = rng.normal(size=(20, 20)) + 1j * rng.normal(size=(20, 20))
    H = (A + A.conj().T) / 2 - .1j * np.diag(np.arange(20))
    x = rng.normal(size=20) + 1j * rng.normal(size=20)
    y, info = cpu_expaction(lambda z: H @ z, x, .3, tol=1e-12)
    save('arnoldi_dense', H=H, x=x, dt=.3, tol=1e-12, y=y, dimension=info['dimension'], exact=expm(-.3j * H) @ x)


def length_gauge_run():
    """A short length-gauge Arnoldi propagation (the cfg-0 method) on a tiny coupled grid:
    midpoint field E(t+dt/2), python/propagate.py:41-50 driven like python/run3d.py:196-199."""
    grid = dict(edges=[0, 1, 2, 3, 4, 5, 6], order=4, ecs_angle=.3, tail=6)
    u = Helium(make_grid(**grid), 2, M=0, cutoff_radii=[2, 3])
    c = CoupledHelium(u, 1)
    op = TorchHamiltonian(c, 'cpu')
    rng = np.random.default_rng(5)
    x = rng.normal(size=c.size) + 1j * rng.normal(size=c.size)
    x /= np.linalg.norm(x)
    pulse = Pulse(omega=1.6, cycles=3, field=.05)
    dt, steps = .05, 6
    states, dims = [x], []
    y = op.state(x)
    from torch_backend import step as torch_step
    for i in range(steps):
        y, info = torch_step(lambda t, v: op.apply(v, (0., 0., float(pulse.electric(t))), False), y, i * dt, dt,
                             tol=1e-11, maxdim=12)
        states.append(op.host(y))
        dims.append(info['dimension'])
    save('length_run', grid=json.dumps(grid), lmax=2, total_Lmax=1, cutoff=np.array([2., 3.]),
         pulse=json.dumps(dict(omega=1.6, cycles=3, field=.05)), dt=dt, tol=1e-11, maxdim=12,
         states=np.array(states), dimensions=np.array(dims))


def cf4_cases():
    # python tests/test_implicit.py:25-35 (separable resolvent) and :67-77 (CF4, both precisions).
    grid = dict(edges=[0, .5, 1, 2, 4], order=3, ecs_angle=.4, tail=6)
    h = Helium(make_grid(**grid), 1, M=None)
    op = TorchHamiltonian(h, 'cpu')
    rng = np.random.default_rng(816)
    xs = rng.normal(size=h.size) + 1j * rng.normal(size=h.size)
    alpha = .02 / (3 + 1j * np.sqrt(3))
    pre = SeparablePreconditioner(op)
    ys = op.host(pre.apply(op.state(xs), alpha, 2.9))
    rng = np.random.default_rng(810)
    x = rng.normal(size=h.size) + 1j * rng.normal(size=h.size)
    x /= np.linalg.norm(x)
    A = lambda t: np.array([.02 * np.cos(t), .01 * np.sin(t), .03])
    answers, infos = {}, {}
    for precision in ('complex128', 'complex64'):
        op.separable = SeparablePreconditioner(op, precision)
        y, info = cf4_step(op, op.state(x), A, 0, .02, -2.9, tol=1e-12)
        answers[precision] = op.host(y)
        infos[precision] = info['linear_iterations']
    # three steps of a z-polarised pulse on a coupled basis
    u = Helium(make_grid(**grid), 2, M=0, cutoff_radii=[1, 2])
    c = CoupledHelium(u, 1)
    cop = TorchHamiltonian(c, 'cpu')
    cop.separable = SeparablePreconditioner(cop)
    rng = np.random.default_rng(11)
    xc = rng.normal(size=c.size) + 1j * rng.normal(size=c.size)
    xc /= np.linalg.norm(xc)
    p = Pulse(omega=1.6, cycles=2, field=.1)
    Az = lambda t: np.array([0., 0., float(p.vector(t))])
    seq = [xc]
    state = cop.state(xc)
    for i in range(3):
        state, _ = cf4_step(cop, state, Az, i * .05, .05, -2.7, tol=1e-11)
        seq.append(cop.host(state))
    save('cf4', grid=json.dumps(grid), lmax=1, x_sep=xs, alpha=alpha, shift=2.9, y_sep=ys, x=x, dt=.02, e_ref=-2.9,
         tol=1e-12, y128=answers['complex128'], y64=answers['complex64'], its128=infos['complex128'],
         its64=infos['complex64'], coupled_lmax=2, coupled_L=1, coupled_cut=np.array([1., 2.]),
         coupled_pulse=json.dumps(dict(omega=1.6, cycles=2, field=.1)), coupled_dt=.05, coupled_e_ref=-2.7,
         coupled_tol=1e-11, coupled_states=np.array(seq))


def gmres_case():
    # python tests/test_implicit.py:57-65.
    rng = np.random.default_rng(31)
    A = np.diag(np.geomspace(1, 1000, 12)).astype(complex)
    A += .03 * (rng.normal(size=A.shape) + 1j * rng.normal(size=A.shape))
    b = rng.normal(size=12) + 1j * rng.normal(size=12)
    pre = torch.tensor(1 / np.diag(A), dtype=torch.complex64)
    x, info = gmres(lambda y: torch.tensor(A) @ y, torch.tensor(b),
                    lambda y: (pre * y.to(torch.complex64)).to(torch.complex128), tol=1e-12, restart=16, flexible=True)
    save('gmres', A=A, b=b, x=x.numpy(), iterations=info['iterations'], solve=np.linalg.solve(A, b))


def volkov_case():
    """Online tSURFF contraction + Volkov accumulation (python/streaming_surface.py:39-64,
    python/surface_contract.py:41-56) on the reference's test configuration
    (tests/test_streaming_surface.py:10-20, linear coupled variant)."""
    from run3d import setup, vector_function
    from streaming_surface import OnlineSurface
    c = {'radial': {'edges': [0, 1, 2, 4, 6, 8], 'order': 3, 'tail': 6, 'ecs_angle': .3},
         'lmax': 1, 'M': 0, 'total_Lmax': 2, 'cutoff_radii': [1, 2], 'surface': 5.,
         'pulses': [{'pulse': {'omega': 5., 'cycles': 2, 'field': .15}, 'polarization': 'z'}],
         'dt': .12, 'post_time': .2, 'ionic_channels': [[1, 0, 0], [2, 0, 0], [2, 1, 0]],
         'spectrum_energy': [.2, 1.2, 7], 'spectrum': {'theta_points': 4, 'phi_points': 1},
         'storage': {'mode': 'spectrum', 'max_file_bytes': 500000, 'ionic_block_frames': 4, 'ionic_device': 'lu'}}
    _, h = setup(c)
    h.prepare_surface(5.)
    A, _ = vector_function(c)
    times = np.linspace(0, 2 * np.pi * 2 / 5, 17)
    with tempfile.TemporaryDirectory() as tmp:
        online = OnlineSurface(h, c, tmp, times, A)
        assert online.prepare()
        contract = online.contract
        rng = np.random.default_rng(424)
        frames = rng.normal(size=(len(times), h.n, len(h.surface_indices), h.nc)) + \
            1j * rng.normal(size=(len(times), h.n, len(h.surface_indices), h.nc))
        chis, qs = [], []
        for i in range(len(times)):
            chi = online.chi_at(i)
            chis.append(chi)
            q = contract(chi, frames[i])
            qs.append(q)
            online.accumulator.add(i, times[i], q)
        acc = online.accumulator
        save('volkov', times=times, avec=np.array([A(t) for t in times]), frames=frames, chi=np.array(chis),
             q=np.array(qs), amplitude=acc.amplitude, tests=acc.tests, harmonics=acc.harmonics, energy=acc.energy,
             theta=acc.theta, phi=acc.phi, solid_angle_weights=acc.solid_angle_weights, unit=acc.unit,
             outerstates=np.array(contract.outerstates), labels=np.array(contract.labels),
             surface_r=h.r[h.surface_indices].real, surface_w=h.grid.weights[h.surface_indices].real,
             transform=h.transform, nion=online.ion.na, n=h.n)
        online.close()


def ground_case():
    # Field-free ground state of a small real grid (python/ground_s.py:55-89).
    grid = dict(edges=[0, .5, 1, 2, 3, 4.5, 6, 8, 10], order=5)
    u = Helium(make_grid(**grid), 2, M=0)
    E, g, res = CoupledHelium(u, 2).ground(tol=1e-10)
    save('ground', grid=json.dumps(grid), lmax=2, energy=E, state=g, residual=res)


def pulses():
    ts = np.linspace(-1, 30, 301)
    arrays = {}
    for k, args in enumerate([dict(omega=1.6, cycles=10, field=.01), dict(omega=1.5, cycles=2.5, field=.02, cep=.7),
                              dict(omega=.9, cycles=3, field=.05, start=2.)]):
        p = Pulse(**args)
        arrays[f'p{k}'] = json.dumps(args)
        arrays[f'p{k}_E'] = p.electric(ts)
        arrays[f'p{k}_A'] = p.vector(ts)
    save('pulses', t=ts, **arrays)


def sharded_case():
    """A (7, 3, 2) complex128 array written frame by frame (in reverse order) through the
    reference's ShardedArray with a 4400-byte cap (three frames per shard, three shards)."""
    import shutil
    from surface_storage import ShardedArray
    folder = Path(__file__).resolve().parent / 'shards'
    if folder.exists():
        shutil.rmtree(folder)
    shape = (7, 3, 2)
    values = (np.arange(np.prod(shape)).reshape(shape) * (1 + 2j) - 3.5j).astype(complex)
    a = ShardedArray(folder, shape, mode='w+', max_file_bytes=4400)
    for i in reversed(range(shape[0])):
        a[i] = values[i]
    a.close()
    save('shards_values', values=values)


def tsurff_run_case():
    """A whole channel-resolved tSURFF run through the reference's own production driver
    (python/run3d.py:_run_impl with the Torch backend on the CPU and online spectrum storage,
    python/streaming_surface.py:OnlineSurface): the small case of laqphysics_b200.tsurff_run
    with post_time 1 a.u., dt 0.02 (the driver rounds it to T / ceil(T / dt)), Krylov
    dimension 16 and tolerance 1e-10.  Stores the spectrum file's arrays, the final state and
    the time grid, so the device run can be compared with the reference's composition of
    propagation, flux, ionic channel functions, contraction and Volkov integral."""
    import run3d
    sys.path.insert(0, str(REPO))
    from laqphysics_b200.tsurff_run import SMALL_CASE
    config = json.loads(json.dumps(SMALL_CASE))
    config.update({'dt': .02, 'post_time': 1.0, 'krylov_dimension': 16, 'krylov_tolerance': 1e-10,
                   'ground_tolerance': 1e-10, 'checkpoint_every': 100000, 'storage': {'mode': 'spectrum'}})
    with tempfile.TemporaryDirectory() as out:
        meta = run3d.run(config, out, backend='torch', device='cpu')
        with np.load(Path(out) / 'spectrum.npz') as d:
            spec = {k: d[k] for k in ('energy', 'theta', 'phi', 'solid_angle_weights', 'amplitudes', 'pes',
                                      'angle_integrated', 'labels')}
        with np.load(Path(out) / 'checkpoint.npz') as d:
            psi, ground = d['psi'], d['ground']
    save('tsurff_run', config=json.dumps(config), dt=meta['dt'], nsteps=meta['nsteps'], ground_energy=meta['ground_energy'],
         psi=psi, ground=ground, **spec)


if __name__ == '__main__':
    if len(sys.argv) > 1:          # named cases only, e.g. `make_golden.py sharded_case`
        for name in sys.argv[1:]:
            globals()[name]()
        sys.exit(0)
    grids()
    product_cases()
    coupled_case()
    bipolar_case()
    ionic_adjoint_case()
    mixed_gauge_case()
    bipolar_contraction_case()
    arnoldi_dense()
    length_gauge_run()
    cf4_cases()
    gmres_case()
    volkov_case()
    ground_case()
    pulses()
    sharded_case()
    tsurff_run_case()
