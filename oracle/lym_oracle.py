"""CPU oracle for the Wilson fermion / SU(N) gauge hot path.

TEST INFRASTRUCTURE ONLY.  This module restates, in plain numpy, the
algorithm of the reference's TensorFlow implementation (emanueleusai/TfLeonardYM,
cited below as ``file:line``) so that the CUDA path can be checked against it.
Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it; the product package
never does.

Pinning: every reference-restating function here is checked against golden
vectors produced by the unmodified reference (``tests/golden/*.npz``, made by
``tests/golden/make_golden.py``) in ``tests/test_oracle_golden.py``.  The
functions marked BUILDER-DEFINED have no reference counterpart (even-odd
preconditioning, CG, multishift CG, exp(i eps H) start links); they are
checked against the reference-restating ones (true residuals, solution
differences), not against reference code.

Layouts are the reference's: spinor (ns, N, V), gauge (nd, N, N, V), complex128,
site index lexicographic with the LAST coordinate fastest.
"""
import numpy as np
import scipy.linalg

# ---------------------------------------------------------------------------
# Lattice runtime
# ---------------------------------------------------------------------------


def lookup_tables(geometry):
    """Neighbour tables and coordinates (lattice.py:86-120).

    Returns (sup, sdn, coords): int64 arrays of shape (nd, V).  Site index is
    the row-major (last coordinate fastest) linearisation of the coordinates.
    """
    geometry = tuple(int(g) for g in geometry)
    nd = len(geometry)
    coords = np.indices(geometry, dtype=np.int64).reshape(nd, -1)
    sup = np.empty_like(coords)
    sdn = np.empty_like(coords)
    for mu in range(nd):
        up = coords.copy()
        up[mu] = (up[mu] + 1) % geometry[mu]
        sup[mu] = np.ravel_multi_index(tuple(up), geometry)
        dn = coords.copy()
        dn[mu] = (dn[mu] - 1) % geometry[mu]
        sdn[mu] = np.ravel_multi_index(tuple(dn), geometry)
    return sup, sdn, coords


def translate(t, tables, mu, sign):
    """Shift along the last (site) axis (lattice.py:124-128)."""
    sup, sdn, _ = tables
    return np.take(t, sup[mu] if sign > 0 else sdn[mu], axis=-1)


def antiperiodic_field(geometry, factor=-1):
    """Per-site factor, ``factor`` on the last time slice (boundary_conditions.py:10-20)."""
    _, _, coords = lookup_tables(geometry)
    f = np.ones(coords.shape[1], dtype=np.complex128)
    f[coords[-1] == geometry[-1] - 1] = factor
    return f


def apply_time_bc(gauge, field):
    """Multiply the last direction's links by the BC field (boundary_conditions.py:23-46)."""
    out = np.array(gauge, dtype=np.complex128, copy=True)
    out[-1] = out[-1] * field[None, None, :]
    return out


# ---------------------------------------------------------------------------
# Dirac operator
# ---------------------------------------------------------------------------


def gammas(nd):
    """Euclidean gamma matrices and gamma_d of the reference basis (dirac.py:284-298)."""
    if nd == 2:
        g = np.array([[[0, 1], [1, 0]], [[0, -1j], [1j, 0]]], dtype=np.complex128)
        gd = np.diag([1, -1]).astype(np.complex128)
    elif nd == 4:
        g = np.array([[[0, 0, 0, -1j], [0, 0, -1j, 0], [0, 1j, 0, 0], [1j, 0, 0, 0]],
                      [[0, 0, 0, -1], [0, 0, 1, 0], [0, 1, 0, 0], [-1, 0, 0, 0]],
                      [[0, 0, -1j, 0], [0, 0, 0, 1j], [1j, 0, 0, 0], [0, -1j, 0, 0]],
                      [[0, 0, 1, 0], [0, 0, 0, 1], [1, 0, 0, 0], [0, 1, 0, 0]]], dtype=np.complex128)
        gd = np.diag([1, 1, -1, -1]).astype(np.complex128)
    elif nd == 3:
        # BUILDER-DEFINED (the reference has no D = 3 fermions, dirac.py:299-300):
        # two-component spinors, gamma_mu = sigma_{mu+1}; no gamma_d exists (odd dimension)
        g = np.array([[[0, 1], [1, 0]], [[0, -1j], [1j, 0]], [[1, 0], [0, -1]]], dtype=np.complex128)
        gd = None
    else:
        raise RuntimeError(f"Number of dimensions {nd} not supported for fermions!")
    return g, gd


def hopping(gauge_bc, psi, tables, dagger=False):
    """H psi = sum_mu U_mu(x)(1-g_mu)psi(x+mu) + U_mu(x-mu)^dag (1+g_mu) psi(x-mu)
    (the hopping sum of dirac.py:503-523, without kappa / identity).  dagger: the
    adjoint hop H^dag, which is H with g_mu -> -g_mu (BUILDER-DEFINED, for D = 3)."""
    nd = gauge_bc.shape[0]
    g, _ = gammas(nd)
    if dagger:
        g = -g
    ident = np.eye(g.shape[1])
    out = np.zeros_like(psi)
    for mu in range(nd):
        fwd = translate(np.einsum("mn,njc->mjc", ident - g[mu], psi), tables, mu, +1)
        out += np.einsum("ijc,mjc->mic", gauge_bc[mu], fwd)
        udn = translate(gauge_bc[mu], tables, mu, -1)
        bwd = translate(np.einsum("mn,njc->mjc", ident + g[mu], psi), tables, mu, -1)
        out += np.einsum("jic,mjc->mic", np.conj(udn), bwd)
    return out


def gamma_d(psi):
    """apply_hermiticity: negate the lower half of the spin components (dirac.py:649-662)."""
    out = np.array(psi, copy=True)
    out[psi.shape[0] // 2:] *= -1
    return out


def wilson_apply(gauge_bc, psi, kappa, hermitian, tables, dagger=False):
    """Fundamental Wilson operator (dirac.py:458-523 + 649-662):
    D psi = psi + kappa * H psi; Q = gamma_d D when hermitian.  dagger: D^dag
    (BUILDER-DEFINED; D = 3 has no hermitian form)."""
    if hermitian and gauge_bc.shape[0] == 3:
        raise RuntimeError("three dimensions have no hermitian form gamma_d D")
    out = psi + kappa * hopping(gauge_bc, psi, tables, dagger)
    return gamma_d(out) if hermitian else out


def wilson_apply_sites(gauge_bc, psi, kappa, hermitian, tables, sites):
    """wilson_apply restricted to the output sites ``sites`` (int array): returns
    (ns, N, len(sites)).  The same formula (dirac.py:503-523 + 649-662) evaluated
    site by site, so that lattices too large for a whole-field numpy apply can be
    checked at a sample of sites."""
    nd = gauge_bc.shape[0]
    g, _ = gammas(nd)
    ident = np.eye(g.shape[1])
    sup, sdn, _ = tables
    sites = np.asarray(sites, dtype=np.int64)
    out = np.array(psi[:, :, sites], dtype=np.complex128, copy=True)
    hop = np.zeros_like(out)
    for mu in range(nd):
        up, dn = sup[mu][sites], sdn[mu][sites]
        fwd = np.einsum("mn,njc->mjc", ident - g[mu], psi[:, :, up])
        hop += np.einsum("ijc,mjc->mic", gauge_bc[mu][:, :, sites], fwd)
        bwd = np.einsum("mn,njc->mjc", ident + g[mu], psi[:, :, dn])
        hop += np.einsum("jic,mjc->mic", np.conj(gauge_bc[mu][:, :, dn]), bwd)
    out = out + kappa * hop
    return gamma_d(out) if hermitian else out


def dot(v1, v2):
    """sum conj(v1) v2 over all indices (algebra_utils.py:5-11)."""
    if v1.shape != v2.shape:
        raise RuntimeError("Incompatible vector shapes!")
    return np.vdot(v1.ravel(), v2.ravel())


# ---------------------------------------------------------------------------
# Solvers (reference semantics)
# ---------------------------------------------------------------------------


def mmmr_multishift(apply, source, shifts, max_steps, precision, omega=0.95):
    """Multishift MMMR (dirac_solver.py:19-53), positive shifts only.

    Base shift = shifts[-1]; absolute stop |<r,r>| < precision.  Returns
    (solutions, step, converged) with ``step`` the value the reference prints.
    """
    if min(shifts) < 0:
        raise NotImplementedError("negative shifts go to BiCGStab in the reference")
    sols = [np.zeros_like(source) for _ in shifts]
    f = [1.0 for _ in shifts]
    r = source.copy()
    step = 0
    for step in range(max_steps):
        p = apply(r) + shifts[-1] * r
        alpha = omega * dot(p, r) / dot(p, p)
        sols[-1] = sols[-1] + alpha * r
        for i, s in enumerate(shifts[:-1]):
            f[i] = f[i] / (1 + (s - shifts[-1]) * alpha)
            sols[i] = sols[i] + alpha * f[i] * r
        r = r - alpha * p
        if abs(dot(r, r)) < precision:
            return sols, step, True
    return sols, step, False


def bicgstab(apply, source, max_steps, precision, initial_guess=None):
    """BiCGStab (dirac_solver.py:61-110): x0 = source (or guess), r0 = x0 - A x0,
    r_hat = x0 + A x0, absolute stop.  Returns (x, step, converged)."""
    x = (source if initial_guess is None else initial_guess).copy()
    ax = apply(x)
    r = x - ax
    rhat = x + ax
    alpha = omega = rho = 1.0
    p = np.zeros_like(source)
    nu = np.zeros_like(source)
    step = 0
    for step in range(max_steps):
        rho_next = dot(rhat, r)
        beta = (rho_next / rho) * (alpha / omega)
        p = r + beta * (p - omega * nu)
        nu = apply(p)
        alpha = rho_next / dot(rhat, nu)
        s = r - alpha * nu
        t = apply(s)
        omega = dot(t, s) / dot(t, t)
        x = x + alpha * p + omega * s
        r = s - omega * t
        if abs(dot(r, r)) < precision:
            return x, step, True
        rho = rho_next
    return x, step, False


# ---------------------------------------------------------------------------
# Gauge side
# ---------------------------------------------------------------------------


def staples(gauge, tables, no_direction=None):
    """Sum of staples per direction (gauge_action.py:56-101, staples.py:23-58).

    S_mu(x) = sum_{nu != mu, nu != no_direction}
      U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag + U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu).
    Directions equal to ``no_direction`` get a zero staple.
    """
    nd = gauge.shape[0]
    out = np.zeros_like(gauge)
    for mu in range(nd):
        if mu == no_direction:
            continue
        for nu in range(nd):
            if nu == mu or nu == no_direction:
                continue
            u_mu_xnu = translate(gauge[mu], tables, nu, +1)
            u_nu_xmu = translate(gauge[nu], tables, mu, +1)
            up = np.einsum("kmc,mnc,pnc->kpc", gauge[nu], u_mu_xnu, np.conj(u_nu_xmu))
            u_nu_dn = translate(gauge[nu], tables, nu, -1)
            u_mu_dn = translate(gauge[mu], tables, nu, -1)
            u_nu_dn_up = translate(u_nu_dn, tables, mu, +1)
            dn = np.einsum("mkc,mnc,npc->kpc", np.conj(u_nu_dn), u_mu_dn, u_nu_dn_up)
            out[mu] += up + dn
    return out


def staple_terms(gauge, tables, no_direction=None):
    """The per-direction lists of per-plane staple terms of staples.py:23-58, in its
    order: for each plane (mu, nu) with mu, nu != no_direction, the up term then the
    down term; an empty list for mu == no_direction."""
    nd = gauge.shape[0]
    out = [[] for _ in range(nd)]
    for mu in range(nd):
        for nu in range(nd):
            if mu == no_direction or nu == no_direction or nu == mu:
                continue
            u_mu_xnu = translate(gauge[mu], tables, nu, +1)
            u_nu_xmu = translate(gauge[nu], tables, mu, +1)
            out[mu].append(np.einsum("kmc,mnc,pnc->kpc", gauge[nu], u_mu_xnu, np.conj(u_nu_xmu)))
            u_nu_dn = translate(gauge[nu], tables, nu, -1)
            u_mu_dn = translate(gauge[mu], tables, nu, -1)
            u_nu_dn_up = translate(u_nu_dn, tables, mu, +1)
            out[mu].append(np.einsum("mkc,mnc,npc->kpc", np.conj(u_nu_dn), u_mu_dn, u_nu_dn_up))
    return out


def gauge_force(gauge, beta, tables):
    """Wilson gauge force (gauge_action.py:13-24,42-53):
    W = U S^dag, F = -beta/(4N) (W^dag - W) with the trace/N removed from the diagonal."""
    nc = gauge.shape[1]
    s = staples(gauge, tables)
    w = np.einsum("mijc,mkjc->mikc", gauge, np.conj(s))
    f = (-0.25 * beta / nc) * (np.conj(np.transpose(w, (0, 2, 1, 3))) - w)
    tr = np.einsum("miic->mc", f) / nc
    for i in range(nc):
        f[:, i, i] -= tr
    return f


def plaquette_trace_sum(gauge, tables):
    """sum_{x, mu<nu} Tr U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag (complex),
    as trace_plaquette (gauge_action.py:110-113) summed over planes."""
    nd = gauge.shape[0]
    total = 0.0
    for mu in range(nd):
        for nu in range(mu + 1, nd):
            u_nu_xmu = translate(gauge[nu], tables, mu, +1)
            u_mu_xnu = translate(gauge[mu], tables, nu, +1)
            total += np.einsum("klc,lmc,nmc,knc", gauge[mu], u_nu_xmu, np.conj(u_mu_xnu), np.conj(gauge[nu]))
    return total


def gauge_energy(gauge, beta, tables):
    """S_g = -beta/N Re sum Tr P (gauge_action.py:26-39)."""
    return -beta * np.real(plaquette_trace_sum(gauge, tables)) / gauge.shape[1]


def plaquette(gauge, tables):
    """<P> = Re sum Tr P / (n_planes N V) (measurements.py:22-43)."""
    nd, nc, _, vol = gauge.shape
    return np.real(plaquette_trace_sum(gauge, tables)) / (nd * (nd - 1) // 2 * nc * vol)


def generators(nc):
    """Fundamental SU(2)/SU(3) generators T^a, Tr T^a T^b = delta/2 (lie_generators.py:3-17)."""
    if nc == 2:
        return np.array([[[0, 1], [1, 0]], [[0, -1j], [1j, 0]], [[1, 0], [0, -1]]], dtype=np.complex128) / 2
    if nc == 3:
        s3 = 1 / np.sqrt(3.0)
        return np.array([
            [[0, 1, 0], [1, 0, 0], [0, 0, 0]], [[0, 0, 1], [0, 0, 0], [1, 0, 0]],
            [[0, 0, 0], [0, 0, 1], [0, 1, 0]], [[0, -1j, 0], [1j, 0, 0], [0, 0, 0]],
            [[0, 0, -1j], [0, 0, 0], [1j, 0, 0]], [[0, 0, 0], [0, 0, -1j], [0, 1j, 0]],
            [[1, 0, 0], [0, -1, 0], [0, 0, 0]], [[s3, 0, 0], [0, s3, 0], [0, 0, -2 * s3]]],
            dtype=np.complex128) / 2
    raise ValueError(nc)


def lie_derivative(gauge_bc, X, Y, kappa, hermitian, tables):
    """Fermion force building block (dirac.py:525-565), fundamental representation.

    Per mu: kappa * sum_k T^k_{ut} [ X^dag P+ T^k U_mu Y(x+mu) - Y(x+mu)^dag P- U_mu^dag T^k X ]
    with P+- = (gamma_d)(1 -+ gamma_mu), gamma_d only when hermitian.
    """
    nd, nc = gauge_bc.shape[0], gauge_bc.shape[1]
    g, gd = gammas(nd)
    ident = np.eye(g.shape[1])
    T = generators(nc)
    out = []
    for mu in range(nd):
        pp = ident - g[mu]
        pm = ident + g[mu]
        if hermitian:
            pp, pm = gd @ pp, gd @ pm
        ysup = translate(Y, tables, mu, +1)
        # A[i,j] = sum_{m,n,l} conj(X)[m,i] P+[m,n] U[j,l] Y(x+mu)[n,l]
        a = np.einsum("mis,mn,jls,nls->ijs", np.conj(X), pp, gauge_bc[mu], ysup)
        # B[j,l] = sum_{m,n,i} conj(Ysup)[m,i] P-[m,n] conj(U)[j,i] X[n,l]
        b = np.einsum("mis,mn,jis,nls->jls", np.conj(ysup), pm, np.conj(gauge_bc[mu]), X)
        d = np.einsum("kij,ijs,kut->uts", T, a, T) - np.einsum("kjl,jls,kut->uts", T, b, T)
        out.append(d)
    return kappa * np.stack(out)


# ---------------------------------------------------------------------------
# Adjoint representation (dirac.py:358-364, 380-456, 525-565; lie_generators.py)
# ---------------------------------------------------------------------------


def adjoint_generators(nc):
    """(T_adj^i)_{jk} = -2 Tr([T_i, T_j] T_k) (lie_generators.py:22-36)."""
    T = generators(nc)
    comm = np.einsum("iab,jbc->ijac", T, T) - np.einsum("jab,ibc->ijac", T, T)
    return -2 * np.einsum("ijab,kba->ijk", comm, T)


def adjoint_vector(psi):
    """Matrix-valued adjoint spinor (ns, N, N, V) -> components (ns, N^2-1, V),
    X_a = 2 Tr(T_a X) (dirac.py:531-532)."""
    T = generators(psi.shape[1])
    return 2 * np.einsum("ijk,mkjc->mic", T, psi)


def adjoint_links(gauge, bc_field=None):
    """V_mu^{ab} = 2 Tr(T_a U_mu T_b U_mu^dag) (dirac.py:358-364), then the
    boundary field on the last direction when given (the provider of dirac.py:368-370)."""
    T = generators(gauge.shape[1])
    v = 2.0 * np.einsum("ijk,mklc,nlo,mjoc->minc", T, gauge, T, np.conj(gauge))
    return apply_time_bc(v, bc_field) if bc_field is not None else v


def adjoint_hopping(gauge_bc, gauge, psi, tables):
    """sum_mu U_mu(x)(1-g_mu)psi(x+mu)U'_mu(x)^dag + U_mu(x-mu)^dag (1+g_mu)psi(x-mu) U'_mu(x-mu)
    for matrix-valued spinors (ns, N, N, V): the left links carry the boundary
    condition, the right ones (the original configuration) do not (dirac.py:380-403)."""
    nd = gauge_bc.shape[0]
    g, _ = gammas(nd)
    ident = np.eye(g.shape[1])
    out = np.zeros_like(psi)
    for mu in range(nd):
        fwd = translate(np.einsum("mn,njkc->mjkc", ident - g[mu], psi), tables, mu, +1)
        out += np.einsum("ijc,mjkc,lkc->milc", gauge_bc[mu], fwd, np.conj(gauge[mu]))
        bwd = translate(np.einsum("mn,njkc->mjkc", ident + g[mu], psi), tables, mu, -1)
        ldn = translate(gauge_bc[mu], tables, mu, -1)
        rdn = translate(gauge[mu], tables, mu, -1)
        out += np.einsum("jic,mjkc,klc->milc", np.conj(ldn), bwd, rdn)
    return out


def wilson_apply_adjoint(gauge_bc, gauge, psi, kappa, hermitian, tables):
    """Adjoint Wilson operator D psi = psi + kappa H psi (Q = gamma_d D when hermitian)."""
    out = psi + kappa * adjoint_hopping(gauge_bc, gauge, psi, tables)
    return gamma_d(out) if hermitian else out


def lie_derivative_adjoint(vlinks, X, Y, kappa, hermitian, tables):
    """dirac.py:525-565 for matrix-valued X, Y: per mu, kappa * sum_k T^k_{ut} [
    Xv^dag P+ T_adj^k V_mu Yv(x+mu) - Yv(x+mu)^dag P- V_mu^dag T_adj^k Xv ] with the
    adjoint components Xv, Yv and the adjoint links V (boundary condition applied)."""
    nd, nc = vlinks.shape[0], X.shape[1]
    g, gd = gammas(nd)
    ident = np.eye(g.shape[1])
    T = generators(nc)
    TA = adjoint_generators(nc)
    xv, yv = adjoint_vector(X), adjoint_vector(Y)
    out = []
    for mu in range(nd):
        pp = ident - g[mu]
        pm = ident + g[mu]
        if hermitian:
            pp, pm = gd @ pp, gd @ pm
        ysup = translate(yv, tables, mu, +1)
        d = np.einsum("mis,mn,kij,jls,nls,kut->uts", np.conj(xv), pp, TA, vlinks[mu], ysup, T)
        d -= np.einsum("mis,mn,jis,kjl,nls,kut->uts", np.conj(ysup), pm, np.conj(vlinks[mu]), TA, xv, T)
        out.append(d)
    return kappa * np.stack(out)


# ---------------------------------------------------------------------------
# Fermion measurements (dirac.py:665-696, fermion_measurements.py:11-115)
# ---------------------------------------------------------------------------


def point_source(site, color, spin, volume, nc, ns, adjoint=False):
    """Unit source at (spin, colour, site); in the adjoint the colour index is a
    generator index and the source is the matrix T^color (fermion_measurements.py:27-38)."""
    if not adjoint:
        v = np.zeros((ns, nc, volume), dtype=np.complex128)
        v[spin, color, site] = 1
        return v
    v = np.zeros((ns, nc, nc, volume), dtype=np.complex128)
    v[spin, :, :, site] = generators(nc)[color]
    return v


def propagator(apply_q, source, tol=1e-26, max_iter=20000):
    """gamma_d Q (Q^2)^-1 source = gamma_d Q^-1 source (dirac.py:670-682 for a Wilson
    operator), with (Q^2)^-1 by CG to |r|^2 <= tol |b|^2."""
    source = np.asarray(source, dtype=np.complex128)
    x = np.zeros_like(source)
    r = source.copy()
    p = r.copy()
    bb = np.vdot(source, source).real
    rr = bb
    for _ in range(max_iter):
        ap = apply_q(apply_q(p))
        a = rr / np.vdot(p, ap).real
        x += a * p
        r -= a * ap
        rn = np.vdot(r, r).real
        if rn <= tol * bb:
            break
        p = r + (rn / rr) * p
        rr = rn
    return gamma_d(apply_q(x))


def pion_correlator(solutions, coords, direction, length, adjoint=False):
    """sum over the solutions of sum_{spin,colour} conj(S) S per site, summed per
    slice of `direction` (fermion_measurements.py:76-90; adjoint: conj(S_cd) S_dc)."""
    corr = np.zeros(length, dtype=np.complex128)
    for s in solutions:
        if adjoint:
            dot = np.einsum("icdm,idcm->m", np.conj(s), s)
        else:
            dot = np.einsum("icm,icm->m", np.conj(s), s)
        for z in range(length):
            corr[z] += dot[coords[direction] == z].sum()
    return corr


# ---------------------------------------------------------------------------
# On-disk gauge format (lattice.py:10-70)
# ---------------------------------------------------------------------------


def read_config_xdr(raw, geometry, nc=3):
    """Decode the reference's XDR configuration (lattice.py:10-70): V x nd x N x (N-1)
    x 2 big-endian float32 (the first N-1 columns of conj(U), re/im, site slowest),
    then nd int32 extents and 3 float64 parameters.  Columns 0 and 1 are
    Gram-Schmidt normalised as the reference does and column 2 = conj(col0 x col1).
    Returns (gauge (nd, N, N, V) complex128, extents, parameters)."""
    raw = np.asarray(raw, dtype=np.uint8).tobytes()
    nd, vol = len(geometry), int(np.prod(geometry))
    n = vol * nd * nc * (nc - 1) * 2
    words = np.frombuffer(raw, dtype=">f4", count=n).astype(np.float64).reshape(vol, nd, nc, nc - 1, 2)
    loaded = words[..., 0] - 1j * words[..., 1]
    out = np.empty((nd, nc, nc, vol), dtype=np.complex128)
    for mu in range(nd):
        c0 = loaded[:, mu, :, 0].T  # (row, V)
        t = 1.0 / np.sqrt(np.abs(c0[0]) ** 2 + np.abs(c0[1]) ** 2 + np.abs(c0[2]) ** 2)
        c0 = c0 * t
        c1 = loaded[:, mu, :, 1].T
        t = c1[0] * np.conj(c0[0]) + c1[1] * np.conj(c0[1]) + c1[2] * np.conj(c0[2])
        c1 = c1 - t * c0
        t = 1.0 / np.sqrt(np.abs(c1[0]) ** 2 + np.abs(c1[1]) ** 2 + np.abs(c1[2]) ** 2)
        c1 = c1 * t
        c2 = np.stack([np.conj(c0[1]) * np.conj(c1[2]) - np.conj(c0[2]) * np.conj(c1[1]),
                       np.conj(c0[2]) * np.conj(c1[0]) - np.conj(c0[0]) * np.conj(c1[2]),
                       np.conj(c0[0]) * np.conj(c1[1]) - np.conj(c0[1]) * np.conj(c1[0])])
        out[mu] = np.stack([c0, c1, c2], axis=1)
    off = 4 * n
    dims = list(np.frombuffer(raw, dtype=">i4", count=nd, offset=off).astype(int))
    params = list(np.frombuffer(raw, dtype=">f8", count=3, offset=off + 4 * nd).astype(float))
    return out, dims, params


# ---------------------------------------------------------------------------
# Gauge observables and smearing (measurements.py:46-330, smearing.py:34-86)
# ---------------------------------------------------------------------------


def path_product(gauge, tables, steps):
    """Per site x, the ordered link product along `steps` starting at x: +(mu+1)
    multiplies U_mu(y) and moves y -> y + mu, -(mu+1) moves y -> y - mu and
    multiplies U_mu(y)^dag.  Returns (N, N, V)."""
    sup, sdn, _ = tables
    nc, vol = gauge.shape[1], gauge.shape[-1]
    y = np.arange(vol)
    m = np.broadcast_to(np.eye(nc, dtype=np.complex128)[..., None], (nc, nc, vol)).copy()
    for st in steps:
        mu = abs(st) - 1
        if st > 0:
            m = np.einsum("ijc,jkc->ikc", m, gauge[mu][..., y])
            y = sup[mu][y]
        else:
            y = sdn[mu][y]
            m = np.einsum("ijc,kjc->ikc", m, np.conj(gauge[mu][..., y]))
    return m


def path_trace(gauge, tables, steps):
    m = path_product(gauge, tables, steps)
    return np.einsum("iic->c", m)


def temporal_plaquette(gauge, tables):
    """Re sum of the (mu, nd-1) plaquette traces / ((nd-1) N V) (measurements.py:46-66)."""
    nd, nc, vol = gauge.shape[0], gauge.shape[1], gauge.shape[-1]
    t = nd - 1
    tot = sum(path_trace(gauge, tables, [mu + 1, t + 1, -(mu + 1), -(t + 1)]).sum() for mu in range(nd - 1))
    return np.real(tot) / ((nd - 1) * nc * vol)


def polyakov_loop_field(gauge, tables, geometry, direction):
    """Trace of the product of the links around the compact `direction` (measurements.py:74-84)."""
    return path_trace(gauge, tables, [direction + 1] * geometry[direction])


def wilson_loops(gauge, tables, d_r, d_t, max_r, max_t):
    """sum_x Tr(R-line T-line R-line^dag T-line^dag) / (N V) for r = 1..max_r,
    t = 1..max_t, in that order (measurements.py:99-140)."""
    nc, vol = gauge.shape[1], gauge.shape[-1]
    out = []
    for r in range(1, max_r + 1):
        for t in range(1, max_t + 1):
            steps = [d_r + 1] * r + [d_t + 1] * t + [-(d_r + 1)] * r + [-(d_t + 1)] * t
            out.append(path_trace(gauge, tables, steps).sum() / (nc * vol))
    return out


def polyakov_operators(gauge, tables, geometry, correlator_direction=2, polyakov_direction=3):
    """(meson zero-momentum projection per slice, Polyakov correlator, Polyakov loop)
    (measurements.py:143-194; the meson pairs P(x) with P(x + e_1))."""
    coords = tables[2]
    p = polyakov_loop_field(gauge, tables, geometry, polyakov_direction)
    meson = p * np.conj(translate(p, tables, 1, +1))
    mz = [meson[(coords[correlator_direction] == z) & (coords[polyakov_direction] == 0)].mean()
          for z in range(geometry[correlator_direction])]
    corr = []
    pdt = p
    for _ in range(geometry[correlator_direction]):
        corr.append((p * np.conj(pdt)).mean())
        pdt = translate(pdt, tables, correlator_direction, +1)
    return np.array(mz), np.array(corr), p.mean()


def glueball_operators(gauge, tables, geometry, correlator_direction=2):
    """Per-slice means of the summed 1x1 and 2x2 plaquette traces over the planes
    that do not contain `correlator_direction` (measurements.py:197-290)."""
    nd = gauge.shape[0]
    coords = tables[2]
    plaq = 0
    square = 0
    for mu in range(nd):
        for nu in range(mu + 1, nd):
            if correlator_direction in (mu, nu):
                continue
            a, b = mu + 1, nu + 1
            plaq = plaq + path_trace(gauge, tables, [a, b, -a, -b])
            square = square + path_trace(gauge, tables, [a, a, b, b, -a, -a, -b, -b])
    length = geometry[correlator_direction]
    pz = np.array([np.mean(plaq[coords[correlator_direction] == z]) for z in range(length)])
    sz = np.array([np.mean(square[coords[correlator_direction] == z]) for z in range(length)])
    return pz, sz


def ape_smearing(gauge, tables, rho, no_smear_direction=3):
    """P_SU(N)[(rho/6) S_mu + (1 - rho) U_mu], S the staples without the
    no-smear direction; a direction without staples keeps rho U_mu + (1 - rho) U_mu
    (smearing.py:34-51)."""
    nd = gauge.shape[0]
    nodir = no_smear_direction if 0 <= no_smear_direction < nd else None
    st = staples(gauge, tables, nodir)
    fat = np.array([(rho / 6) * st[mu] if mu != nodir else rho * gauge[mu] for mu in range(nd)])
    return unitary_sqrt_projection(fat + (1 - rho) * gauge)


def update_link_field(links, momenta, eps):
    """U <- expm(eps P) U per link (hmc.py:40-43)."""
    ex = scipy.linalg.expm(np.transpose(eps * momenta, (0, 3, 1, 2)))  # (nd, V, N, N)
    return np.einsum("mcij,mjkc->mikc", ex, links)


def update_momenta(momenta, force, eps):
    """P <- P + eps F (hmc.py:59-61)."""
    return momenta + eps * force


def momenta_energy(momenta):
    """K = -Re sum Tr P^2 (hmc.py:170-176)."""
    return -np.real(np.einsum("mijc,mjic->", momenta, momenta))


def unitary_sqrt_projection(x):
    """X (X^dag X)^{-1/2} / det^{1/N} per link (smearing.py:17-31), principal roots."""
    nd, nc, _, vol = x.shape
    m = np.transpose(x, (0, 3, 1, 2))  # (nd, V, N, N)
    h = np.conj(np.swapaxes(m, -1, -2)) @ m
    w, v = np.linalg.eigh(h)
    inv_sqrt = (v * (1.0 / np.sqrt(w))[..., None, :]) @ np.conj(np.swapaxes(v, -1, -2))
    u = m @ inv_sqrt
    det = np.linalg.det(u)
    u = u / (det ** (1.0 / nc))[..., None, None]
    return np.transpose(u, (0, 2, 3, 1))


def random_momenta_from_normals(normals, nc):
    """Anti-Hermitian traceless momenta from unit normals, as hmc.py:69-96 builds them.

    ``normals`` has shape (nd, nc*nc - 1, V): for each direction, the
    off-diagonal (real, imag) pairs in the order (i<j), then the nc-1 Cartan
    values; each is scaled by 1/2 as in the reference.
    """
    nd, _, vol = normals.shape
    p = np.zeros((nd, nc, nc, vol), dtype=np.complex128)
    for mu in range(nd):
        k = 0
        for i in range(nc):
            for j in range(i + 1, nc):
                re, im = normals[mu, k] / 2, normals[mu, k + 1] / 2
                k += 2
                p[mu, i, j] = re + 1j * im
                p[mu, j, i] = -re + 1j * im
        diag = np.zeros((nc, vol))
        for i in range(1, nc):
            r = normals[mu, k] / 2
            k += 1
            for j in range(i):
                diag[j] += r / np.sqrt(i * (i + 1) / 2.0)
            diag[i] += -r * (i * np.sqrt(2.0 / (i * (i + 1))))
        for i in range(nc):
            p[mu, i, i] = 1j * diag[i]
    return p


# ---------------------------------------------------------------------------
# Fermion action (Nf=2 with R(Q^2) = sum alpha_i (Q^2 + beta_i)^-1)
# ---------------------------------------------------------------------------


class WilsonSetup:
    """Bundle of (gauge with BC applied, kappa, tables) for the action helpers."""

    def __init__(self, gauge, kappa, geometry, bc_factor=-1, hermitian=True):
        self.tables = lookup_tables(geometry)
        self.geometry = tuple(geometry)
        self.kappa = kappa
        self.hermitian = hermitian
        self.bc_field = antiperiodic_field(geometry, bc_factor) if bc_factor is not None else None
        self.set_gauge(gauge)

    def set_gauge(self, gauge):
        self.gauge = gauge
        self.gauge_bc = apply_time_bc(gauge, self.bc_field) if self.bc_field is not None else gauge

    def Q(self, v):
        return wilson_apply(self.gauge_bc, v, self.kappa, self.hermitian, self.tables)

    def Q2(self, v):
        return self.Q(self.Q(v))


def fermion_force(setup, phi, alphas, betas, solve):
    """n_flavor.force (fermion_action.py:64-93): X_i = (Q^2+beta_i)^-1 phi, Y_i = Q X_i,
    F = sum_i alpha_i [L(X_i, Y_i) + L(Y_i, X_i)]."""
    xs = solve(setup.Q2, phi, betas)
    f = 0
    for x, a in zip(xs, alphas):
        y = setup.Q(x)
        f = f + a * (lie_derivative(setup.gauge_bc, x, y, setup.kappa, setup.hermitian, setup.tables)
                     + lie_derivative(setup.gauge_bc, y, x, setup.kappa, setup.hermitian, setup.tables))
    return f


def fermion_energy(setup, phi, alphas, betas, solve, shift=0.0):
    """n_flavor.energy (fermion_action.py:39-44) with RationalApproximation.apply (dirac.py:52-59)."""
    xs = solve(setup.Q2, phi, betas)
    r = shift * phi
    for x, a in zip(xs, alphas):
        r = r + a * x
    return np.real(dot(phi, r))


def integrate_om(gauge, momenta, force_fns, steps, delta_t, level=0):
    """Nested Omelyan integrator (hmc.py:133-162).

    ``force_fns[i](gauge)`` returns the force of action i; the innermost level
    moves the links.  Returns (gauge, momenta).
    """
    ll = 0.19318332275037863
    eps = delta_t / steps[level]
    last = level == len(force_fns) - 1
    momenta = update_momenta(momenta, force_fns[level](gauge), -ll * eps)
    force = None
    for _ in range(steps[level]):
        if last:
            gauge = update_link_field(gauge, momenta, eps / 2)
        else:
            gauge, momenta = integrate_om(gauge, momenta, force_fns, steps, eps / 2, level + 1)
        force = force_fns[level](gauge)
        momenta = update_momenta(momenta, force, -(1 - 2 * ll) * eps)
        if last:
            gauge = update_link_field(gauge, momenta, eps / 2)
        else:
            gauge, momenta = integrate_om(gauge, momenta, force_fns, steps, eps / 2, level + 1)
        force = force_fns[level](gauge)
        momenta = update_momenta(momenta, force, -2 * ll * eps)
    momenta = update_momenta(momenta, force, +ll * eps)
    return gauge, momenta


# ---------------------------------------------------------------------------
# BUILDER-DEFINED: even-odd preconditioning and CG (no reference counterpart)
# ---------------------------------------------------------------------------


def parity_maps(geometry):
    """Even-odd maps.  parity(x) = sum_i x_i mod 2; within a parity sites keep
    lexicographic order, so the checkerboard index is lex // 2 (all extents even).
    Returns (parity (V,), cb (V,), eo_to_lex (2, V/2))."""
    geometry = tuple(geometry)
    if any(g % 2 for g in geometry):
        raise ValueError("even-odd ordering needs even extents")
    _, _, coords = lookup_tables(geometry)
    par = coords.sum(axis=0) % 2
    lex = np.arange(coords.shape[1])
    cb = lex // 2
    eo = np.empty((2, coords.shape[1] // 2), dtype=np.int64)
    for p in (0, 1):
        eo[p, cb[par == p]] = lex[par == p]
    return par, cb, eo


def to_eo(v, eo):
    return v[..., eo[0]], v[..., eo[1]]


def from_eo(ve, vo, eo):
    out = np.empty(ve.shape[:-1] + (2 * ve.shape[-1],), dtype=ve.dtype)
    out[..., eo[0]] = ve
    out[..., eo[1]] = vo
    return out


def cg_normal(apply_a, apply_adag, b, tol_abs_res, max_iter, x0=None):
    """Textbook CGNR on A^dag A x = A^dag b, stopping on the TRUE residual
    |b - A x| < tol_abs_res (recomputed whenever the recursive one passes)."""
    x = np.zeros_like(b) if x0 is None else x0.copy()
    r_true = b - apply_a(x)
    r = apply_adag(r_true)
    p = r.copy()
    rr = np.real(dot(r, r))
    it = 0
    while it < max_iter:
        t = apply_a(p)
        alpha = rr / np.real(dot(t, t))
        x = x + alpha * p
        r = r - alpha * apply_adag(t)
        rr_new = np.real(dot(r, r))
        it += 1
        if rr_new < (0.1 * tol_abs_res) ** 2:
            res = np.linalg.norm(b - apply_a(x))
            if res < tol_abs_res:
                return x, it, res
        p = r + (rr_new / rr) * p
        rr = rr_new
    return x, it, np.linalg.norm(b - apply_a(x))


def eo_solve(setup, b, tol=1e-10, max_iter=20000):
    """Solve D x = b (D = 1 + kappa H, the reference sign) by even-odd Schur
    preconditioning M = 1 - kappa^2 H_eo H_oe and CGNR.  Returns (x, iters, rel_true_res)."""
    par, cb, eo = parity_maps(setup.geometry)
    k = setup.kappa

    def hop_full(v):
        return hopping(setup.gauge_bc, v, setup.tables)

    def h_eo(vo):  # even output from odd input
        full = from_eo(np.zeros_like(vo), vo, eo)
        return hop_full(full)[..., eo[0]]

    def h_oe(ve):
        full = from_eo(ve, np.zeros_like(ve), eo)
        return hop_full(full)[..., eo[1]]

    def m(ve):
        return ve - k * k * h_eo(h_oe(ve))

    def mdag(ve):
        return gamma_d(m(gamma_d(ve)))

    be, bo = to_eo(b, eo)
    bp = be - k * h_eo(bo)
    bnorm = np.linalg.norm(b)
    xe, it, _ = cg_normal(m, mdag, bp, tol * bnorm, max_iter)
    xo = bo - k * h_oe(xe)
    x = from_eo(xe, xo, eo)
    d = x + k * hop_full(x)
    return x, it, np.linalg.norm(b - d) / bnorm


def multishift_cg(apply, b, shifts, tol, max_iter):
    """BUILDER-DEFINED multishift CG on (A + sigma_s) x_s = b for Hermitian
    positive A (recurrences of Jegerlehner, hep-lat/9612014).  The base system
    is the smallest shift; the others follow through the zeta recurrences.
    Stops when every shift's residual |r_s| = |zeta_s| |r| is below tol*|b|.
    Returns (xs, iterations)."""
    n = len(shifts)
    base = int(np.argmin(shifts))
    s0 = shifts[base]
    x = [np.zeros_like(b) for _ in range(n)]
    p = [b.copy() for _ in range(n)]
    r = b.copy()
    rr = np.real(dot(r, r))
    stop2 = tol * tol * rr
    z_prev = np.ones(n)
    z = np.ones(n)
    a_prev, b_prev = 1.0, 0.0
    active = np.ones(n, bool)
    it = 0
    while it < max_iter:
        ap = apply(p[base]) + s0 * p[base]
        a = rr / np.real(dot(p[base], ap))
        z_next = np.ones(n)
        for s in range(n):
            if not active[s]:
                continue
            if s == base:
                x[s] = x[s] + a * p[s]
                continue
            d = shifts[s] - s0
            z_next[s] = z[s] * z_prev[s] * a_prev / (
                a * b_prev * (z_prev[s] - z[s]) + z_prev[s] * a_prev * (1.0 + d * a))
            x[s] = x[s] + (a * z_next[s] / z[s]) * p[s]
        r = r - a * ap
        rr_new = np.real(dot(r, r))
        bet = rr_new / rr
        for s in range(n):
            if not active[s]:
                continue
            if s == base:
                p[s] = r + bet * p[s]
            else:
                p[s] = z_next[s] * r + bet * (z_next[s] / z[s]) ** 2 * p[s]
        it += 1
        for s in range(n):
            if s != base and active[s] and z_next[s] ** 2 * rr_new < stop2:
                active[s] = False
        z_prev, z = z, np.where(active | (np.arange(n) == base), z_next, z)
        a_prev, b_prev, rr = a, bet, rr_new
        if rr_new < stop2:
            break
    return x, it
