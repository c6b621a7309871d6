"""Input validation of ``unwrap()``.

The exception types and messages are part of the drop-in: callers and the
reference's test suite match on them (test_unwrap.py:44-80: "cost must be",
"init must be", "2-D", "shape", "complex", "floating").  The rules are kept
in two tables -- one predicate per dtype family, one set of choices per
string option -- and every public checker is a thin call into them.
"""
import numpy as np

_MASK_DTYPES = (np.dtype("bool"), np.dtype("uint8"), np.dtype("int8"))

# dtype family -> (accepts(dtype), what the message says the array must be)
_DTYPE_RULES = {
    "complex": (lambda dt: np.issubdtype(dt, np.complexfloating), "complex"),
    "float": (lambda dt: np.issubdtype(dt, np.floating), "floating-point"),
    "integer": (lambda dt: np.issubdtype(dt, np.integer), "integer"),
    "mask": (lambda dt: dt in _MASK_DTYPES, "bool or 8-bit integer"),
}

# string option -> accepted values
_CHOICES = {
    "cost": frozenset(("smooth", "defo", "topo")),
    "init": frozenset(("mst", "mcf", "laplace")),
}


def _dtype_of(arr):
    """dtype without reading a dataset that declares one"""
    dt = getattr(arr, "dtype", None)
    return np.dtype(dt) if dt is not None else np.asarray(arr).dtype


def _require_dtype(family, arrays):
    accepts, what = _DTYPE_RULES[family]
    for name, arr in arrays.items():
        dt = _dtype_of(arr)
        if not accepts(dt):
            raise TypeError(f"{name} must be {what}, got dtype={dt}")


def _require_choice(option, value):
    valid = set(_CHOICES[option])
    if value not in valid:
        raise ValueError(f"{option} must be one of {valid}, got {value!r}")


def check_2d_shape(arr, name):
    """(nrow, ncol) of ``arr``; ValueError unless it is 2-D."""
    ndim = np.ndim(arr)
    if ndim != 2:
        raise ValueError(f"{name} must be 2-D, got ndim={ndim}")
    shape = np.shape(arr)
    return int(shape[0]), int(shape[1])


def check_shape_match(ref_shape, **arrays):
    """ValueError naming the first array whose shape is not ``ref_shape``."""
    for name, arr in arrays.items():
        shape = np.shape(arr)
        if shape != ref_shape:
            raise ValueError(f"{name} shape {shape} does not match expected {ref_shape}")


def check_complex_dtype(**arrays):
    _require_dtype("complex", arrays)


def check_float_dtype(**arrays):
    _require_dtype("float", arrays)


def check_integer_dtype(**arrays):
    _require_dtype("integer", arrays)


def check_bool_or_byte_dtype(**arrays):
    _require_dtype("mask", arrays)


def check_cost_mode(cost):
    _require_choice("cost", cost)


def check_init_method(init):
    _require_choice("init", init)
