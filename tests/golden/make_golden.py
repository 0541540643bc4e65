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
    """The jax.numpy calls used by the reference's _apply_toeplitz, on numpy."""

    @staticmethod
    def asarray(x):
        return np.asarray(x, dtype=np.float64).view(_Updatable)

    def __getattr__(self, name):
        fn = getattr(np, name)

        def wrapped(*args, **kwargs):
            out = fn(*args, **kwargs)
            return out.view(_Updatable) if isinstance(out, np.ndarray) else out

        return wrapped


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
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
