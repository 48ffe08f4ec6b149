"""Start-up of a stop-fit worker process (run with runpy.run_path by the
spawned pool in earlystop.start_fit_pool): this package importable under its
own name, since it is loaded from its folder rather than installed and a
spawned process starts without it, the fits' modules imported, and one BLAS
thread per worker.  The limit is set through threadpoolctl after the imports:
the parent's main module is re-imported in a spawned child before this runs,
so NumPy's BLAS can already be loaded with one thread per core, and workers
that each spin that many BLAS threads slow the fits down by an order of
magnitude."""
import importlib.util
import os
import sys

for _v in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS"):
    os.environ[_v] = "1"

_NAME = "special_topics_b200"
if _NAME not in sys.modules:
    _dir = os.path.dirname(os.path.abspath(__file__))
    _spec = importlib.util.spec_from_file_location(_NAME, os.path.join(_dir, "__init__.py"),
                                                   submodule_search_locations=[_dir])
    _mod = importlib.util.module_from_spec(_spec)
    sys.modules[_NAME] = _mod
    _spec.loader.exec_module(_mod)

import scipy.linalg  # noqa: E402,F401
import scipy.optimize  # noqa: E402,F401
from threadpoolctl import threadpool_limits  # noqa: E402

threadpool_limits(limits=1)
