"""Generate the golden fixtures in tests/golden/ by running the reference's own code.

The reference (licongxu/GMaster) is a JAX package and JAX is not installed here, so the
package cannot be imported as a whole.  Its pure-numpy helpers can still be run: this
script parses the reference source files, extracts the named functions/classes with
``ast`` and executes exactly that source with numpy in scope.  The outputs (together
with the seeded inputs) are saved as small ``.npz`` fixtures that travel with the repo;
the tests never read the reference at run time.

Run from the repository root (needs the reference checkout):

    python tests/golden/make_golden.py /root/reference

Fixtures written:
  geometry.npz   gmaster/utils.py:_SHTInfo (theta, phi0, nphi, offsets) for several Nside,
                 and gmaster/_sht/rings.py:_ring_czt_constants_numpy (nphi, start).
  bins.npz       gmaster/bins.py:_linear_bands for several (lmax, nlb).
  coupling_tt.npz  tests/test_workspaces.py:_shrinking_offset_tt on seeded windows, and
                 _triangle_cuda_indexing (float64 and float32-product arms).
  toeplitz.npz   gmaster/workspaces.py:_apply_toeplitz on exact scalar couplings and on a
                 random symmetric matrix, and _toeplitz_exact_pairs.  _apply_toeplitz is
                 written against jax.numpy's functional updates (``x.at[i].set(v)``); it is
                 run here with numpy behind a minimal stand-in for those calls.
  quadrature.npz gmaster/workspaces.py:_wigner_d_table and _general_coupling_matrix_quadrature
                 (with the tables of _wigner_d_triple, the spin-0 x 2 and 2 x 2 blocks of
                 _coupling_matrices_spin2 and the general spins of the workspace builder) on
                 seeded mask spectra.  ducc0 is absent, so the Gauss-Legendre nodes and
                 weights are the oracle's (saved beside the outputs); jax.lax.scan, jax.jit and
                 gammaln are run through numpy / scipy stand-ins.
  slots.npz      the (block, row channel, column channel, sign) table that the workspace
                 builder (gmaster/workspaces.py, NmtWorkspace coupling assembly, the code
                 from "blocks = []" up to _assemble_mcm) produces for each spin pair,
                 executed with a stand-in workspace object.
  spectra_eb.npz gmaster/workspaces.py:_compute_coupled_cell on seeded alms; the E/B
                 combination of gmaster/_sht/healpix.py:_map2alm_once_impl applied to the
                 oracle's spin-s transform of Q + iU at every order (the s2fft forward
                 transform it calls is absent and is replaced by that array); and
                 gmaster/_sht/healpix.py:_unpack_spin on seeded E/B alms.
"""

import ast
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def extract(path, names, extra_globals=None):
    """Execute only the top-level definitions `names` of a source file; return them."""
    with open(path) as handle:
        tree = ast.parse(handle.read(), filename=path)
    wanted = [node for node in tree.body
              if isinstance(node, (ast.FunctionDef, ast.ClassDef)) and node.name in names]
    missing = set(names) - {node.name for node in wanted}
    if missing:
        raise KeyError(f"{path}: missing {sorted(missing)}")
    module = ast.Module(body=wanted, type_ignores=[])
    from functools import lru_cache, partial

    namespace = {"np": np, "jnp": None, "lru_cache": lru_cache, "partial": partial}
    if extra_globals:
        namespace.update(extra_globals)
    exec(compile(module, path, "exec"), namespace)
    return {name: namespace[name] for name in names}


class _Updatable(np.ndarray):
    """numpy array with jax-style functional updates: ``x.at[index].set(values)``."""

    @property
    def at(self):
        array = self

        class _Index:
            def __getitem__(self, index):
                class _Setter:
                    def set(self, values):
                        out = np.array(array, copy=True)
                        out[index] = values
                        return out.view(_Updatable)

                return _Setter()

        return _Index()


class _NumpyAsJnp:
    """The jax.numpy calls used by the extracted reference functions, on numpy (float64
    unless the input says otherwise; `precision=` keywords of matmul are dropped)."""

    @staticmethod
    def asarray(x, dtype=None):
        out = np.asarray(x, dtype=dtype)
        if dtype is None and out.dtype.kind in "iub":
            out = out.astype(np.float64)
        return out.view(_Updatable)

    @staticmethod
    def matmul(a, b, precision=None):
        return np.matmul(a, b).view(_Updatable)

    def __getattr__(self, name):
        fn = getattr(np, name)
        if not callable(fn) or isinstance(fn, type):
            return fn

        def wrapped(*args, **kwargs):
            out = fn(*args, **kwargs)
            return out.view(_Updatable) if isinstance(out, np.ndarray) else out

        return wrapped


class _JaxStandIn:
    """jax.jit (identity), jax.lax.scan (a loop), jax.vmap and jax.ops.segment_sum on numpy."""

    @staticmethod
    def jit(fn=None, **kwargs):
        return fn if fn is not None else (lambda f: f)

    @staticmethod
    def vmap(fn):
        return lambda xs: np.stack([fn(x) for x in xs]).view(_Updatable)

    class lax:  # noqa: N801 - mirrors the module name
        class Precision:
            HIGHEST = None

        @staticmethod
        def scan(fn, carry, xs, unroll=1):
            ys = []
            for x in xs:
                carry, y = fn(carry, x)
                ys.append(y)
            if not ys:   # an empty scan stacks nothing: shape (0, *carry item)
                return carry, np.zeros((0,) + np.shape(carry[-1])).view(_Updatable)
            return carry, np.stack(ys).view(_Updatable)

    class ops:  # noqa: N801
        @staticmethod
        def segment_sum(data, ids, num_segments):
            return np.bincount(np.asarray(ids), weights=np.asarray(data), minlength=num_segments)


class _ConfigStandIn:
    @staticmethod
    def make_room(nbytes):
        return None


def main(ref_root):
    utils = os.path.join(ref_root, "gmaster", "utils.py")
    rings = os.path.join(ref_root, "gmaster", "_sht", "rings.py")
    bins = os.path.join(ref_root, "gmaster", "bins.py")
    tws = os.path.join(ref_root, "tests", "test_workspaces.py")

    sht_info = extract(utils, ["_SHTInfo"])["_SHTInfo"]
    czt = extract(rings, ["_ring_czt_constants_numpy"])["_ring_czt_constants_numpy"]
    geometry = {}
    for nside in (1, 2, 4, 8, 16, 32, 64, 256, 2048):
        info = sht_info(nside)
        geometry[f"theta_{nside}"] = info.theta
        geometry[f"phi0_{nside}"] = info.phi0
        geometry[f"nphi_{nside}"] = info.nphi.astype(np.int64)
        geometry[f"offsets_{nside}"] = info.offsets.astype(np.int64)
        geometry[f"weight_{nside}"] = np.float64(info.weight)
        if nside >= 2:
            L = 3 * nside
            nphi, start = czt(L, nside)[:2]
            geometry[f"czt_nphi_{nside}"] = np.asarray(nphi).astype(np.int64)
            geometry[f"czt_start_{nside}"] = np.asarray(start).astype(np.int64)
    np.savez_compressed(os.path.join(HERE, "geometry.npz"), **geometry)

    linear = extract(bins, ["_linear_bands"])["_linear_bands"]
    bands = {}
    for lmax, nlb in ((191, 16), (47, 4), (50, 7), (6143, 16), (23, 1), (10, 16)):
        ells, bpws = linear(lmax, nlb)
        bands[f"ells_{lmax}_{nlb}"] = ells.astype(np.int64)
        bands[f"bpws_{lmax}_{nlb}"] = bpws.astype(np.int64)
    np.savez_compressed(os.path.join(HERE, "bins.npz"), **bands)

    fns = extract(tws, ["_shrinking_offset_tt", "_triangle_cuda_indexing"])
    coupling = {}
    for lmax in (15, 16, 17, 31, 40):
        window = np.random.default_rng(20 + lmax).uniform(size=2 * lmax + 1)
        coupling[f"window_{lmax}"] = window
        coupling[f"tt_{lmax}"] = fns["_shrinking_offset_tt"](window, lmax)
    window = np.random.default_rng(23).uniform(size=2 * 24 + 1)
    coupling["window_tri"] = window
    coupling["tri64"] = fns["_triangle_cuda_indexing"](window, 24, use_f32=False)
    coupling["tri32"] = fns["_triangle_cuda_indexing"](window, 24, use_f32=True)
    np.savez_compressed(os.path.join(HERE, "coupling_tt.npz"), **coupling)

    ws = os.path.join(ref_root, "gmaster", "workspaces.py")
    toe = extract(ws, ["_apply_toeplitz", "_toeplitz_exact_pairs"], {"jnp": _NumpyAsJnp()})
    toeplitz = {}
    cases = [(31, 16, 4, 3), (40, 20, 5, 2), (12, 6, 3, 2), (25, 10, 10, 0), (30, 28, 1, 4)]
    with np.errstate(divide="ignore", invalid="ignore"):
        for k, (lmax, lt, le, db) in enumerate(cases):
            window = np.random.default_rng(40 + k).uniform(size=2 * lmax + 1)
            cols = 2 * np.arange(lmax + 1) + 1
            S = fns["_shrinking_offset_tt"](window, lmax) / cols[None]
            toeplitz[f"case_{k}"] = np.array([lmax, lt, le, db], dtype=np.int64)
            toeplitz[f"window_{k}"] = window
            toeplitz[f"S_{k}"] = S
            toeplitz[f"out_{k}"] = np.asarray(toe["_apply_toeplitz"](S, lt, le, db))
            rows, columns = toe["_toeplitz_exact_pairs"](lmax + 1, lt, le, db)
            toeplitz[f"pairs_{k}"] = np.stack([rows, columns], 1).astype(np.int64)
        rng = np.random.default_rng(50)
        A = rng.uniform(0.1, 1.0, size=(20, 20))
        A = A + A.T
        toeplitz["random_S"] = A
        toeplitz["random_out"] = np.asarray(toe["_apply_toeplitz"](A, 9, 2, 3))
    np.savez_compressed(os.path.join(HERE, "toeplitz.npz"), **toeplitz)

    quadrature_and_slots(ref_root)
    spectra_and_eb(ref_root)
    print("wrote", sorted(os.listdir(HERE)))


def _oracle():
    root = os.path.dirname(os.path.dirname(HERE))
    if root not in sys.path:
        sys.path.insert(0, root)
    import oracle

    oracle.build()
    return oracle


# Spin cases of the quadrature fixture: (s1, s2, n1, n2).  The spin-0 x 2 and 2 x 2 blocks
# are those of _coupling_matrices_spin2; the rest are the workspace builder's general spins.
QUAD_CASES = [(0, 2, 0, 2), (2, 2, 2, 2), (0, 0, 0, 0), (0, 1, 0, 1), (1, 0, 1, 0), (1, 1, 1, 1),
              (1, 3, 1, 3), (3, 3, 3, 3), (0, 3, 0, 3), (2, 1, 2, 1)]
# Wigner-d tables of the fixture: (m, n) pairs of those triples and a few more.
WIGNER_PAIRS = [(0, 0), (2, 2), (-2, -2), (0, 2), (0, -2), (2, -2), (1, 3), (-1, -3), (3, -1),
                (1, 0), (0, 4), (4, 4)]
# Workspaces of the slot fixture: (spin1, spin2, is_teb).
SLOT_CASES = [(0, 0, False), (0, 2, False), (2, 0, False), (2, 2, False), (0, 2, True),
              (0, 1, False), (1, 0, False), (1, 3, False), (3, 3, False), (0, 3, True), (1, 1, False)]


def quadrature_and_slots(ref_root):
    from scipy.special import gammaln

    orc = _oracle()
    ws = os.path.join(ref_root, "gmaster", "workspaces.py")
    jnp = _NumpyAsJnp()
    names = ["_wigner_d_table", "_general_coupling_matrix_quadrature", "_wigner_d_shared",
             "_wigner_d_triple"]
    fns = extract(ws, names, {"jnp": jnp, "jax": _JaxStandIn, "gammaln": gammaln,
                              "_config": _ConfigStandIn, "_coupling_f32": lambda lmax: False,
                              "_WD_TRIPLE_CACHE": {}})
    quad = {}
    lmax = 12
    lmax_mask = 2 * lmax
    order = (2 * lmax + lmax_mask) // 2 + 1
    nodes, weights = orc.gauss_legendre(order)
    beta = np.arccos(nodes)
    quad["lmax"] = np.int64(lmax)
    quad["lmax_mask"] = np.int64(lmax_mask)
    quad["nodes"] = nodes
    quad["weights"] = weights
    for m, n in WIGNER_PAIRS:
        quad[f"wigner_{m}_{n}"] = np.asarray(fns["_wigner_d_table"](beta, m=m, n=n, lmax=lmax_mask))
    for k, (s1, s2, n1, n2) in enumerate(QUAD_CASES):
        window = np.random.default_rng(60 + k).uniform(0.1, 1.0, size=lmax_mask + 1)
        window /= (1.0 + np.arange(lmax_mask + 1)) ** 2
        tables = fns["_wigner_d_triple"](beta, s1=s1, s2=s2, n1=n1, n2=n2, lmax=lmax,
                                         lmax_mask=lmax_mask)
        out = fns["_general_coupling_matrix_quadrature"](window, weights, tables, lmax=lmax,
                                                         lmax_mask=lmax_mask)
        tag = f"{s1}_{s2}_{n1}_{n2}"
        quad[f"window_{tag}"] = window
        quad[f"blocks_{tag}"] = np.asarray(out)
    np.savez_compressed(os.path.join(HERE, "quadrature.npz"), **quad)

    # the slot table of the workspace builder, run on a stand-in workspace with the block
    # names in place of the blocks
    with open(ws) as handle:
        lines = handle.read().split("\n")
    start = next(i for i, t in enumerate(lines) if t.strip() == "blocks = []")
    stop = next(i for i in range(start, len(lines)) if lines[i].strip() == "_drop_large_wigner_cache()")
    body = "\n".join(t[8:] for t in lines[start:stop])
    slots = {}
    for k, (s1, s2, teb) in enumerate(SLOT_CASES):
        ncls = 7 if teb else (1 if s1 == s2 == 0 else (2 if s1 == 0 or s2 == 0 else 4))

        class Workspace:
            pass

        ws_obj = Workspace()
        ws_obj.ncls, ws_obj.spin1, ws_obj.spin2 = ncls, s1, s2
        ws_obj.pure_e1 = ws_obj.pure_b1 = ws_obj.pure_e2 = ws_obj.pure_b2 = False
        env = {"self": ws_obj, "scalar": "tt", "te": "te", "even": "even", "odd": "odd",
               "pure_any": False}
        exec(compile(body, ws, "exec"), env)
        names_idx = {"tt": 0, "te": 1, "even": 2, "odd": 3}
        table = np.array([[names_idx[b], r, c, sg] for b, (r, c), sg in
                          zip(env["blocks"], env["slots"], env["signs"])], dtype=np.int64)
        slots[f"case_{k}"] = np.array([s1, s2, int(teb), ncls], dtype=np.int64)
        slots[f"table_{k}"] = table
    np.savez_compressed(os.path.join(HERE, "slots.npz"), **slots)


def spectra_and_eb(ref_root):
    orc = _oracle()
    ws = os.path.join(ref_root, "gmaster", "workspaces.py")
    hp = os.path.join(ref_root, "gmaster", "_sht", "healpix.py")
    jnp = _NumpyAsJnp()
    out = {}
    cell = extract(ws, ["_compute_coupled_cell"], {"jnp": jnp, "jax": _JaxStandIn})["_compute_coupled_cell"]
    lmax = 13
    L = lmax + 1
    ell = np.concatenate([np.arange(m, L) for m in range(L)])
    order = np.repeat(np.arange(L), L - np.arange(L))
    rng = np.random.default_rng(70)
    for n1, n2 in ((1, 1), (2, 1), (2, 2)):
        a1 = rng.normal(size=(n1, len(ell))) + 1j * rng.normal(size=(n1, len(ell)))
        a2 = rng.normal(size=(n2, len(ell))) + 1j * rng.normal(size=(n2, len(ell)))
        a1[:, order == 0] = a1[:, order == 0].real
        a2[:, order == 0] = a2[:, order == 0].real
        out[f"alm1_{n1}{n2}"], out[f"alm2_{n1}{n2}"] = a1, a2
        out[f"cl_{n1}{n2}"] = np.asarray(cell(a1, a2, ell, order, lmax=lmax))

    # E/B combination of the analysis, fed the oracle's spin-s transform of Q + iU
    nside = 4
    lmax_eb = 3 * nside - 1
    Le = lmax_eb + 1
    ell_e = np.concatenate([np.arange(m, Le) for m in range(Le)])
    order_e = np.repeat(np.arange(Le), Le - np.arange(Le))
    plus_box = {}
    once = extract(hp, ["_map2alm_once_impl"], {
        "jnp": jnp, "jax": _JaxStandIn,
        "_forward_s2fft_impl": lambda *a, **k: plus_box["plus"].view(_Updatable)})["_map2alm_once_impl"]
    unpack = extract(hp, ["_unpack_spin", "_packed_triangle"], {"jnp": jnp, "jax": _JaxStandIn})
    for spin in (1, 2, 3):
        qu = np.random.default_rng(80 + spin).normal(size=(2, 12 * nside ** 2))
        plus = orc.spin_plus(qu, spin, nside, lmax_eb)
        plus_box["plus"] = plus
        eb = once(qu, (), ell_e, order_e, spin=spin, nside=nside, L=Le, L_work=Le)
        out[f"qu_s{spin}"] = qu
        out[f"plus_s{spin}"] = plus
        out[f"eb_s{spin}"] = np.asarray(eb)
        ebr = rng.normal(size=(2, len(ell_e))) + 1j * rng.normal(size=(2, len(ell_e)))
        ebr[:, order_e == 0] = ebr[:, order_e == 0].real
        ebr[:, ell_e < spin] = 0
        out[f"ebin_s{spin}"] = ebr
        out[f"unpack_s{spin}"] = np.asarray(unpack["_unpack_spin"](ebr, Le, Le))
    np.savez_compressed(os.path.join(HERE, "spectra_eb.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
