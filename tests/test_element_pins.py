"""Independent pins of the element constructions behind the qubit-mode (Jaynes-Cummings),
optomechanics (CoupledModes N-X) and qubit-chain (CoupledModes X-X in RWA) workloads.

The golden runs of the reference pin the PTLA, the mode and the particle elements, but no
golden run contains a Jaynes-Cummings coupling, a qubit treated as a two-level mode, or a
CoupledModes interaction.  Here the operators of those systems are built as dense matrices
directly from the reference's formulas, with numpy and nothing of this library's element
code:

  mode   H/i = -z n + eta a^+ - eta* a  (Sch, z = kappa - i delta; Mode.cc:56-86, Mode.tcc:184-193)
         IP: H/i = eta a^+ - eta* a furnished with frequencies, Exact part exp(-zI n t)
         (Mode.cc:42-45,94-99, Mode.tcc:170-177), zI = kappa - i delta
         jump sqrt(2 kappa) a, rate 2 kappa <n> (Mode.cc:118-125, Mode_.h:180-184)
         averages <n>, <n^2>, Re<a>, Im<a> (Mode.cc:177-196)
  qubit  the mode form on dimension 2 with -eta (Qbit_.h:100-116, Qbit.cc:86-165),
         jump sqrt(2 gamma) sigma (Qbit.cc:38-42), averages rho00, rho11, Re/Im rho10
         (Qbit.cc:22-32)
  JC     H/i = g* sigma a^+ - g sigma^+ a (JaynesCummings_.h:54-66)
  CM_NX  H/i = Re(u) n (a + a^+)/sqrt(2) / i, CM_XX_RWA  H/i = u* a1 a2^+ - u a1^+ a2
         (CoupledModes.cc:20-41, Mode_.h:38); Optomechanics passes u -> -sqrt(2) u
         (Optomechanics.cc:36-38)

In the interaction picture an off-diagonal entry (out, in) of a free element's H/i carries
the phase exp(tau (lambda[out] - lambda[in])), lambda = zI n the Exact exponents
(Tridiagonal::furnishWithFreqs / propagate, Tridiagonal.cc:24-36, Tridiagonal.tcc:153-163),
i.e. E(tau)^-1 H0/i E(tau) with E(tau) = exp(-lambda tau).  An interaction is a direct
product of one-axis operators, and the reference composes its frequencies by a direct sum
of the factors' frequency arrays (Tridiagonal.tcc:56-64) in which an empty array (a main
diagonal, or a factor of an element without an Exact part) empties the product
(ComplexArrayExtensions.h:80-95): an entry keeps its phase only when it is off-diagonal on
every factor's axis and every factor's element is in an Exact picture.  So the N-X coupling
n (a + a^+) of optomechanics stays time-independent in the interaction picture, as in the
reference.  The product's descriptor (the Tridiagonal
terms of cqg_model_create) is compared with these matrices: the Hamiltonian through the
oracle's slice-wise apply, the Exact exponents, the jump operators and rate weights and
the observables through a numpy reading of the descriptor's documented diagonal
numbering, all on random states to 1e-13.
"""
import ctypes as C

import numpy as np
import pytest

from cppqed_b200 import _abi as A

TOL = 1e-13


# ---- dense reference operators ------------------------------------------------------

def lowering(N):
    return np.diag(np.sqrt(np.arange(1, N, dtype=float)), 1).astype(complex)  # a|n> = sqrt(n)|n-1>


def number(N):
    return np.diag(np.arange(N, dtype=float)).astype(complex)


def dag(X):
    return X.conj().T


class Free:
    """A free element: H/i without the Exact part, Exact exponents lambda[n], jumps, rate
    weights and its averages as a function of the reduced density matrix."""

    def __init__(self, N, H0, lam, jumps, weights, averages):
        self.N, self.H0, self.lam, self.jumps, self.weights, self.averages = N, H0, lam, jumps, weights, averages


def mode_averages(rho):
    N = rho.shape[0]
    n = np.arange(N)
    off = sum(np.sqrt(k) * rho[k, k - 1] for k in range(1, N))  # Tr(rho a)
    return [np.sum(n * rho.diagonal().real), np.sum(n * n * rho.diagonal().real), off.real, off.imag]


def qbit_averages(rho):
    return [rho[0, 0].real, rho[1, 1].real, rho[1, 0].real, rho[1, 0].imag]


def two_level_mode(N, kappa, delta, eta, picture, averages):
    """The reference's pumped lossy mode on N levels (the qubit is N = 2 with -eta)."""
    a, n = lowering(N), number(N)
    pump = eta * dag(a) - np.conj(eta) * a
    if picture == "Sch":
        H0 = -(kappa - 1j * delta) * n + pump
        lam = None
    else:
        H0 = pump
        lam = (kappa - 1j * delta) * np.arange(N)
    jumps, weights = [], []
    if kappa:
        jumps.append(np.sqrt(2 * kappa) * a)
        weights.append(2 * kappa * np.arange(N, dtype=float))
    return Free(N, H0, lam, jumps, weights, averages)


def mode(N, kappa, delta, eta, picture):
    return two_level_mode(N, kappa, delta, eta, picture, mode_averages)


def qbit(gamma, delta, eta, picture):
    return two_level_mode(2, gamma, delta, -eta, picture, qbit_averages)


def embed(ops, dims):
    """Kronecker product with axis 0 most significant; ops maps axis -> matrix."""
    out = np.ones((1, 1), dtype=complex)
    for a, N in enumerate(dims):
        out = np.kron(out, ops.get(a, np.eye(N)))
    return out


class Composite:
    def __init__(self, frees, interactions):
        self.frees = frees
        self.dims = [f.N for f in frees]
        self.D = int(np.prod(self.dims))
        self.idx = np.array(np.unravel_index(np.arange(self.D), self.dims))
        # terms: (matrix, axes whose factors must be off-diagonal and furnished for a phase)
        self.terms = [(embed({a: f.H0}, self.dims), [a]) for a, f in enumerate(frees)]
        for axes, factors in interactions:
            for coef, mats in factors:
                self.terms.append((coef * embed(dict(zip(axes, mats)), self.dims), list(axes)))
        lam = np.zeros(self.D, dtype=complex)
        self.has_exact = False
        for a, f in enumerate(frees):
            if f.lam is not None:
                self.has_exact = True
                lam += f.lam[self.idx[a]]
        self.lam = lam

    def hamiltonian(self, tau):
        H = np.zeros((self.D, self.D), dtype=complex)
        for T, axes in self.terms:
            keep = np.ones((self.D, self.D), dtype=bool)
            expo = np.zeros((self.D, self.D), dtype=complex)
            for a in axes:
                lam = self.frees[a].lam
                out, inn = self.idx[a][:, None], self.idx[a][None, :]
                keep &= (out != inn) & (lam is not None)
                if lam is not None:
                    expo += lam[out] - lam[inn]
            H += np.where(keep, T * np.exp(tau * expo), T)
        return H

    def jumps(self):
        out = []
        for a, f in enumerate(self.frees):
            for J, w in zip(f.jumps, f.weights):
                out.append((embed({a: J}, self.dims), a, w))
        return out

    def averages(self, psi):
        t = psi.reshape(self.dims)
        cols = []
        for a, f in enumerate(self.frees):
            m = np.moveaxis(t, a, 0).reshape(self.dims[a], -1)
            cols += f.averages(m @ m.conj().T)
        return np.array(cols)


def jc(g):
    """(axes, [(coefficient, per-axis matrices)]) of g* sigma a^+ - g sigma^+ a on (qubit, mode)."""
    def make(Nq, Nm):
        s, a = lowering(Nq), lowering(Nm)
        return [(np.conj(g), [s, dag(a)]), (-g, [dag(s), a])]
    return make


# ---- reading the product's descriptor (cqg.h: diagonal numbering and boxes) -----------

def term_dense(dims, t, tau=0.0):
    """Dense matrix of a cqg_tridiagonal placed on axes of a system of extents dims:
    diagonal j = sum_a digit_a 3^(rank-1-a); digit 0 main (out n <- in n), 1 minus
    (out n+K <- in n), 2 plus (out n <- in n+K); coefficients C-order over the box,
    times exp(tau freq) where frequencies are given."""
    R = t.rank
    axes = [t.axes[a] for a in range(R)]
    K = [t.differences[a] for a in range(R)]
    sub = [dims[x] for x in axes]
    Dsub = int(np.prod(sub))
    A_ = np.zeros((Dsub, Dsub), dtype=complex)
    for j in range(3 ** R):
        if not t.diagonals[j]:
            continue
        digits = [(j // 3 ** (R - 1 - a)) % 3 for a in range(R)]
        ext = [sub[a] if digits[a] == 0 else sub[a] - K[a] for a in range(R)]
        n = int(np.prod(ext))
        vals = np.array([complex(t.diagonals[j][c].re, t.diagonals[j][c].im) for c in range(n)])
        if t.freqs and t.freqs[j]:
            fr = np.array([complex(t.freqs[j][c].re, t.freqs[j][c].im) for c in range(n)])
            vals = vals * np.exp(tau * fr)
        for c, m in enumerate(np.ndindex(*ext)):
            out = [m[a] + (K[a] if digits[a] == 1 else 0) for a in range(R)]
            inn = [m[a] + (K[a] if digits[a] == 2 else 0) for a in range(R)]
            A_[np.ravel_multi_index(out, sub), np.ravel_multi_index(inn, sub)] += vals[c]
    # embed: identity on the other axes
    D = int(np.prod(dims))
    idx = np.array(np.unravel_index(np.arange(D), dims))
    subidx = np.ravel_multi_index(idx[axes], sub)
    others = [a for a in range(len(dims)) if a not in axes]
    key = np.ravel_multi_index(idx[others], [dims[a] for a in others]) if others else np.zeros(D, dtype=int)
    same = key[:, None] == key[None, :]
    return np.where(same, A_[subidx[:, None], subidx[None, :]], 0)


def descriptor(model):
    d = model.desc.contents
    dims = [d.dims[a] for a in range(d.rank)]
    return d, dims


# ---- the systems --------------------------------------------------------------------

def cplx(z):
    """A complex parameter in the reference's "(re,im)" syntax."""
    z = complex(z)
    return "(%r,%r)" % (z.real, z.imag)


def qbitmode(picture, deltaA, gamma, deltaC, kappa, eta, N, g, etat=0.0):
    args = ["--picture", picture, "--deltaA", str(deltaA), "--gamma", str(gamma), "--deltaC", str(deltaC),
            "--kappa", str(kappa), "--eta", cplx(eta), "--cutoff", str(N), "--g", cplx(g), "--etat", cplx(etat)]
    ref = Composite([qbit(gamma, deltaA, etat, picture), mode(N, kappa, deltaC, eta, picture)],
                    [((0, 1), jc(g)(2, N))])
    return "QbitMode_C++QED", args, ref


def optomechanics(picture, No, Nm, etaO, kappaO, deltaO, kappaM, deltaM, u):
    args = ["--picture", picture, "--cutoffOpt", str(No), "--cutoffMech", str(Nm), "--etaOpt", str(etaO),
            "--kappaOpt", str(kappaO), "--deltaCOpt", str(deltaO), "--kappaMech", str(kappaM),
            "--deltaCMech", str(deltaM), "--u", str(u)]
    uref = -np.sqrt(2) * u
    x = (lowering(Nm) + dag(lowering(Nm))) / np.sqrt(2)
    ref = Composite([mode(No, kappaO, deltaO, etaO, picture), mode(Nm, kappaM, deltaM, 0.0, picture)],
                    [((0, 1), [(uref / 1j, [number(No), x])])])
    return "Optomechanics", args, ref


def qbit_chain(picture, n, gamma, deltaA, etat, u):
    args = ["--picture", picture, "--nQbit", str(n), "--gamma", str(gamma), "--deltaA", str(deltaA),
            "--etat", cplx(etat), "--u", cplx(u)]
    frees = [qbit(gamma, deltaA, etat if i == 0 else 0.0, picture) for i in range(n)]
    s = lowering(2)
    inter = [((i, i + 1), [(np.conj(u), [s, dag(s)]), (-u, [dag(s), s])]) for i in range(n - 1)]
    return "QbitChain", args, Composite(frees, inter)


SYSTEMS = {
    # the headline qubit-mode workload and detuned / driven / complex-coupling variants
    "qbitmode_c2_sch": qbitmode("Sch", 0.0, 0.5, 0.0, 1.0, 1.5, 40, 2 + 0j),
    "qbitmode_detuned_sch": qbitmode("Sch", -1.3, 0.5, 2.1, 0.7, 1.5 - 0.4j, 12, 1.7 - 0.6j, etat=0.3 + 0.2j),
    "qbitmode_detuned_ip": qbitmode("IP", -1.0, 0.5, 2.0, 1.0, 1.5, 40, 2 + 0j),
    "qbitmode_driven_ip": qbitmode("IP", -1.3, 0.5, 2.1, 0.7, 1.5 - 0.4j, 12, 1.7 - 0.6j, etat=0.3 + 0.2j),
    "qbitmode_lossless_qbit_ip": qbitmode("IP", 0.8, 0.0, -0.5, 1.0, 1.0, 10, 3 + 0j),
    # optomechanics (CM_NX), the serving library's 15 x 30 and an interaction-picture case
    "optomechanics_sch": optomechanics("Sch", 15, 30, 2.0, 1.0, -1.0, 0.1, -2.0, 0.2),
    "optomechanics_ip": optomechanics("IP", 4, 12, 1.0, 1.0, -1.0, 0.3, -2.0, 0.1),
    # 6-qubit chain with nearest-neighbour CM_XX_RWA couplings
    "qbit_chain_sch": qbit_chain("Sch", 6, 0.4, -0.7, 0.9 + 0.1j, 0.8 - 0.3j),
    "qbit_chain_ip": qbit_chain("IP", 4, 0.4, -0.7, 0.9 + 0.1j, 0.8 - 0.3j),
}


def random_states(n, D, seed):
    rng = np.random.default_rng(seed)
    psi = rng.normal(size=(n, D)) + 1j * rng.normal(size=(n, D))
    return psi / np.linalg.norm(psi, axis=1, keepdims=True)


@pytest.fixture(scope="module", params=sorted(SYSTEMS))
def system(request, engine):
    script, args, ref = SYSTEMS[request.param]
    model = engine.Model(script, args)
    return request.param, model, ref


def test_dimensions_and_picture(system):
    name, model, ref = system
    d, dims = descriptor(model)
    assert dims == ref.dims
    assert model.dim == ref.D


@pytest.mark.parametrize("tau", [0.0, 0.37, -1.1])
def test_hamiltonian_matches_reference_formulas(system, oracle, tau):
    """H/i(tau) psi through the oracle's slice-wise Tridiagonal apply of the descriptor
    against the dense operator built from the reference's formulas."""
    name, model, ref = system
    H = ref.hamiltonian(tau)
    for psi in random_states(3, ref.D, 11):
        got = oracle.apply_hamiltonian(model, psi, tau)
        want = H @ psi
        assert np.linalg.norm(got - want) <= TOL * max(np.linalg.norm(want), 1.0), name


def test_descriptor_hamiltonian_terms_match(system):
    """The same through a numpy reading of the descriptor's Tridiagonal terms (no oracle)."""
    name, model, ref = system
    d, dims = descriptor(model)
    for tau in (0.0, 0.53):
        H = sum(term_dense(dims, d.ham[i], tau) for i in range(d.n_ham))
        assert np.abs(H - ref.hamiltonian(tau)).max() <= TOL * max(np.abs(H).max(), 1.0), name


def test_exact_part_matches(system):
    name, model, ref = system
    d, dims = descriptor(model)
    lam = np.zeros(ref.D, dtype=complex)
    any_exact = False
    for a in range(d.rank):
        if d.exact[a]:
            any_exact = True
            la = np.array([complex(d.exact[a][n].re, d.exact[a][n].im) for n in range(dims[a])])
            lam += embed({a: np.diag(la)}, dims).diagonal()
    if not any_exact:  # an Exact part with all exponents zero is no Exact part
        assert np.abs(ref.lam).max() == 0
    # the descriptor holds the exponent of U(tau) = exp(-zI n tau) (cqg.h), i.e. -lambda
    assert np.abs(lam + ref.lam).max() <= TOL * max(np.abs(ref.lam).max(), 1.0)


def test_jumps_and_rate_weights_match(system):
    """Jump operators in the reference's ordinal order (frees in axis order) and their
    closed-form rates sum_n w_n |psi_n|^2 = ||J psi||^2."""
    name, model, ref = system
    d, dims = descriptor(model)
    want = ref.jumps()
    assert d.n_jumps == len(want)
    psis = random_states(4, ref.D, 5)
    for m, (J, axis, w) in enumerate(want):
        jd = d.jumps[m]
        got = term_dense(dims, jd.op)
        assert np.abs(got - J).max() <= TOL * np.abs(J).max(), (name, m)
        assert jd.rate_weights, (name, m)
        assert jd.rate_axis == axis
        wd = np.array([jd.rate_weights[n] for n in range(dims[axis])])
        assert np.allclose(wd, w, rtol=TOL, atol=TOL)
        wfull = embed({axis: np.diag(wd.astype(complex))}, dims).diagonal().real
        for psi in psis:
            assert abs(np.sum(wfull * np.abs(psi) ** 2) - np.linalg.norm(J @ psi) ** 2) <= 1e-12


def test_observables_match_reduced_density_averages(system):
    """Linear average columns <psi|O|psi> of the descriptor against the elements' average_v
    of the reduced density matrices (frees in axis order, BinarySystem.cc:141-156)."""
    name, model, ref = system
    d, dims = descriptor(model)
    for psi in random_states(3, ref.D, 7):
        cols = np.zeros(d.n_avr)
        for k in range(d.n_obs):
            o = d.obs[k]
            if o.dense:
                a = o.dense_axis
                N = dims[a]
                M = np.array([complex(o.dense[i].re, o.dense[i].im) for i in range(N * N)]).reshape(N, N)
                Op = embed({a: M}, dims)
            else:
                Op = term_dense(dims, o.op)
            v = psi.conj() @ Op @ psi
            if o.col_re >= 0:
                cols[o.col_re] += v.real
            if o.col_im >= 0:
                cols[o.col_im] += v.imag
        want = ref.averages(psi)
        assert cols.shape == want.shape, name
        assert np.allclose(cols, want, rtol=1e-12, atol=TOL), (name, cols, want)
