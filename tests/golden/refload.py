"""Load the reference's own CPU path (Python 2 + Numba sources) under Python 3.

Used only by ``make_golden.py`` in a checkout where the reference sources are
present; nothing on the GPU side imports it.  The sources are read where they
lie, a few Python-2-only constructs are rewritten in memory, and the results
are registered in ``sys.modules`` under the names the reference imports them
by.  No reference source is copied into this repository.

In-memory rewrites (each one a syntax or Python-2-semantics fix, none changes
the algorithm):
  * the trailing ``if __name__ == '__main__':`` demo blocks are dropped
    (they use Python 2 ``print`` statements);
  * integer ``/`` in index arithmetic becomes ``//``
    (MyML/MyML/EAC/sparse.py:1087, MyML/MyML/utils/sorting.py:21);
  * ``np.argmin(map(len, ensemble))`` gets a ``list(...)``
    (MyML/MyML/EAC/sparse.py:157), since a ``map`` object is not a sequence;
  * implicit relative imports resolve through module aliases;
  * ``tables``/``matplotlib`` are stubbed, ``xrange``/``np.float``/``np.int``
    are provided; the dense-EAC modules (``full``, ``MyML.cluster`` linkage)
    are stubbed because the sparse path never calls them.
"""
import builtins
import os
import sys
import types

os.environ.setdefault("NUMBA_ENABLE_CUDASIM", "1")  # K_Means creates CUDA events

import numpy as np


def _reference_root():
    """The reference checkout, named by the EAC_REFERENCE_ROOT variable (no
    default: the fixtures are only regenerated where the reference is)."""
    root = os.environ.get("EAC_REFERENCE_ROOT")
    if not root:
        raise RuntimeError("set EAC_REFERENCE_ROOT to the reference checkout "
                           "(the directory holding MyML/ and scipy_numba/)")
    return root


REF = _reference_root()

_REWRITES = {
    "MyML/MyML/EAC/sparse.py": [
        ("imid = (imax + imin) / 2", "imid = (imax + imin) // 2"),
        ("np.argmin(map(len,ensemble))", "np.argmin(list(map(len,ensemble)))"),
    ],
    "MyML/MyML/utils/sorting.py": [
        ("mid_arg = args[(r+w) / 2]", "mid_arg = args[(r+w) // 2]"),
    ],
}


def _stub(name, **attrs):
    m = types.ModuleType(name)
    m.__dict__.update(attrs)
    sys.modules[name] = m
    return m


def _load(relpath, modname, aliases=()):
    path = os.path.join(REF, relpath)
    with open(path) as f:
        src = f.read()
    for old, new in _REWRITES.get(relpath, []):
        assert old in src, (relpath, old)
        src = src.replace(old, new)
    lines = src.split("\n")
    for i, line in enumerate(lines):
        if line.startswith("if __name__ =="):
            lines = lines[:i]
            break
    src = "\n".join(lines)
    mod = types.ModuleType(modname)
    mod.__file__ = path
    sys.modules[modname] = mod
    for a in aliases:
        sys.modules[a] = mod
    exec(compile(src, path, "exec"), mod.__dict__)
    return mod


_loaded = None


def load():
    """Return a namespace with the reference's hot-path entry points."""
    global _loaded
    if _loaded is not None:
        return _loaded
    builtins.xrange = range
    if not hasattr(np, "float"):
        np.float = float
    if not hasattr(np, "int"):
        np.int = int
    _stub("tables")
    mpl = _stub("matplotlib")
    mpl.pyplot = _stub("matplotlib.pyplot")
    for pkg in ("MyML", "MyML.utils", "MyML.graph", "MyML.EAC",
                "scipy_numba", "scipy_numba.sparse", "scipy_numba.sparse.csgraph",
                "scipy_numba.spatial"):
        m = _stub(pkg)
        m.__path__ = []
    scan = _load("MyML/MyML/utils/scan.py", "MyML.utils.scan")
    sorting = _load("MyML/MyML/utils/sorting.py", "MyML.utils.sorting")
    kmeans = _load("MyML/MyML/cluster/KMeans.py", "MyML.cluster.KMeans", ["KMeans"])
    _stub("MyML.cluster", KMeans=kmeans.K_Means, SL=None, clusters_from_SL=None,
          __path__=[])
    partition = _load("MyML/MyML/utils/partition.py", "MyML.utils.partition")
    mst = _load("MyML/MyML/graph/mst.py", "MyML.graph.mst", ["mst"])
    cc = _load("MyML/MyML/graph/connected_components.py",
               "MyML.graph.connected_components")
    kruskal = _load("scipy_numba/scipy_numba/sparse/csgraph/_min_spanning_tree.py",
                    "scipy_numba.sparse.csgraph._min_spanning_tree")
    _stub("scipy_numba.spatial.distance", squareform=None)
    sparse = _load("MyML/MyML/EAC/sparse.py", "MyML.EAC.sparse", ["sparse"])
    _stub("full", EAC_FULL=None)
    eac = _load("MyML/MyML/EAC/eac.py", "MyML.EAC.eac")
    rules = _load("MyML/MyML/EAC/rules.py", "MyML.EAC.rules", ["rules"])
    _loaded = types.SimpleNamespace(scan=scan, sorting=sorting, kmeans=kmeans,
                                    partition=partition, mst=mst, cc=cc,
                                    kruskal=kruskal, sparse=sparse, eac=eac,
                                    rules=rules)
    return _loaded
