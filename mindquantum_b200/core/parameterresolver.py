"""ParameterResolver: a linear combination ``const + sum_i coeff_i * p_i`` of named parameters.

Mirrors the reference ``mindquantum.core.parameterresolver.ParameterResolver``
(mindquantum/core/parameterresolver/parameterresolver.py:95-1203) for the part the
state-vector path uses: construction from a str / number / dict, arithmetic,
encoder/ansatz flags, requires-grad flags and ``combination`` (evaluation).

Every parameter of a gate is a ParameterResolver.  The device lowering turns it
into ``angle = const + sum_j coeff_j * params[index_j]`` so the Jacobi of the
reference (ccsrc/lib/math/pr/parameter_resolver.cpp:560-573) is just ``coeff_j``.
"""
from __future__ import annotations

import numbers
from typing import Dict, Iterable, Union

import numpy as np

PRConvertible = Union[str, numbers.Number, Dict[str, numbers.Number], "ParameterResolver"]


class ParameterResolver:
    """A parameter expression ``const + sum coeff * name``.

    Args:
        data: ``None``, a parameter name, a number (the constant), a dict
            ``{name: coeff}`` or another ParameterResolver.
        const: extra constant added to the expression.
        dtype: accepted for interface compatibility; values are kept as Python numbers.
    """

    def __init__(self, data=None, const=None, dtype=None):  # pylint: disable=unused-argument
        self._data: Dict[str, numbers.Number] = {}
        self._const: numbers.Number = 0.0
        self._encoder: set = set()
        self._no_grad: set = set()
        if isinstance(data, ParameterResolver):
            self._data = dict(data._data)
            self._const = data._const
            self._encoder = set(data._encoder)
            self._no_grad = set(data._no_grad)
        elif isinstance(data, str):
            self._data[data] = 1.0
        elif isinstance(data, numbers.Number):
            self._const = data
        elif isinstance(data, dict):
            for k, v in data.items():
                if not isinstance(k, str):
                    raise TypeError(f"Parameter name should be a string, but get {type(k)}.")
                if not isinstance(v, numbers.Number):
                    raise TypeError(f"Parameter value should be a number, but get {type(v)}.")
                self._data[k] = v
        elif isinstance(data, np.ndarray) and data.size == 1:
            self._const = data.item()
        elif data is not None:
            raise TypeError(f"Cannot build a ParameterResolver from {type(data)}.")
        if const is not None:
            self._const = self._const + const

    # ------------------------------------------------------------------ container protocol
    def __len__(self):
        return len(self._data)

    def __contains__(self, key):
        return key in self._data

    def __iter__(self):
        return iter(list(self._data.keys()))

    def __getitem__(self, key):
        return self._data[key]

    def __setitem__(self, key, value):
        if not isinstance(key, str):
            raise TypeError(f"Parameter name should be a string, but get {type(key)}.")
        self._data[key] = value

    def keys(self):
        return iter(list(self._data.keys()))

    def values(self):
        return iter(list(self._data.values()))

    def items(self):
        return iter(list(self._data.items()))

    def pop(self, key):
        self._encoder.discard(key)
        self._no_grad.discard(key)
        return self._data.pop(key)

    # ------------------------------------------------------------------ properties
    @property
    def const(self):
        return self._const

    @const.setter
    def const(self, value):
        self._const = value

    @property
    def params_name(self):
        return list(self._data.keys())

    @property
    def params_value(self):
        return list(self._data.values())

    @property
    def encoder_parameters(self):
        return [k for k in self._data if k in self._encoder]

    @property
    def ansatz_parameters(self):
        return [k for k in self._data if k not in self._encoder]

    @property
    def no_grad_parameters(self):
        return [k for k in self._data if k in self._no_grad]

    @property
    def requires_grad_parameters(self):
        return [k for k in self._data if k not in self._no_grad]

    @property
    def is_complex(self):
        vals = list(self._data.values()) + [self._const]
        return any(isinstance(v, complex) and v.imag != 0 for v in vals)

    def is_const(self):
        return not self._data

    # ------------------------------------------------------------------ flags
    def as_encoder(self):
        self._encoder = set(self._data.keys())
        return self

    def as_ansatz(self):
        self._encoder = set()
        return self

    def encoder_part(self, *names):
        for n in names:
            if n not in self._data:
                raise KeyError(f"Parameter {n} not in this parameter resolver.")
            self._encoder.add(n)
        return self

    def ansatz_part(self, *names):
        for n in names:
            if n not in self._data:
                raise KeyError(f"Parameter {n} not in this parameter resolver.")
            self._encoder.discard(n)
        return self

    def no_grad(self):
        self._no_grad = set(self._data.keys())
        return self

    def requires_grad(self):
        self._no_grad = set()
        return self

    def no_grad_part(self, *names):
        for n in names:
            if n not in self._data:
                raise KeyError(f"Parameter {n} not in this parameter resolver.")
            self._no_grad.add(n)
        return self

    def requires_grad_part(self, *names):
        for n in names:
            if n not in self._data:
                raise KeyError(f"Parameter {n} not in this parameter resolver.")
            self._no_grad.discard(n)
        return self

    # ------------------------------------------------------------------ arithmetic
    def _copy_flags_from(self, *others):
        for o in others:
            if isinstance(o, ParameterResolver):
                self._encoder |= o._encoder
                self._no_grad |= o._no_grad
        return self

    def __copy__(self):
        return ParameterResolver(self)

    def __deepcopy__(self, memo):
        return ParameterResolver(self)

    def copy(self):
        return ParameterResolver(self)

    def __neg__(self):
        out = ParameterResolver(self)
        out._data = {k: -v for k, v in out._data.items()}
        out._const = -out._const
        return out

    def __add__(self, other: PRConvertible):
        other = other if isinstance(other, ParameterResolver) else ParameterResolver(other)
        out = ParameterResolver(self)
        for k, v in other._data.items():
            out._data[k] = out._data.get(k, 0) + v
        out._const = out._const + other._const
        return out._copy_flags_from(other)

    __radd__ = __add__

    def __sub__(self, other: PRConvertible):
        other = other if isinstance(other, ParameterResolver) else ParameterResolver(other)
        return self + (-other)

    def __rsub__(self, other: PRConvertible):
        return (-self) + other

    def __mul__(self, other):
        if isinstance(other, ParameterResolver):
            if other.is_const():
                other = other.const
            elif self.is_const():
                return other * self.const
            else:
                raise ValueError("Product of two non-constant parameter resolvers is not linear.")
        out = ParameterResolver(self)
        out._data = {k: v * other for k, v in out._data.items()}
        out._const = out._const * other
        return out

    __rmul__ = __mul__

    def __truediv__(self, other):
        return self * (1.0 / other)

    def __eq__(self, other):
        other = other if isinstance(other, ParameterResolver) else ParameterResolver(other)
        return self._data == other._data and self._const == other._const

    def __hash__(self):
        return id(self)

    def __float__(self):
        if not self.is_const():
            raise ValueError("Parameter resolver is not a constant.")
        return float(np.real(self._const))

    def __bool__(self):
        return bool(self._data) or self._const != 0

    # ------------------------------------------------------------------ evaluation
    def combination(self, other):
        """Evaluate ``const + sum coeff * other[name]``; returns a ParameterResolver constant.

        Mirrors ``ParameterResolver.combination`` (parameterresolver.py:741-767).
        """
        other = other if isinstance(other, ParameterResolver) else ParameterResolver(other)
        val = self._const
        for k, v in self._data.items():
            if k not in other._data:
                raise ValueError(f"Parameter {k} not in given parameter resolver.")
            val = val + v * other._data[k]
        return ParameterResolver(val)

    def subs(self, other):
        other = other if isinstance(other, ParameterResolver) else ParameterResolver(other)
        out = ParameterResolver(self)
        for k in list(out._data.keys()):
            if k in other._data:
                out._const = out._const + out._data.pop(k) * other._data[k]
                out._encoder.discard(k)
                out._no_grad.discard(k)
        return out

    def expression(self):
        terms = [f"{v}*{k}" for k, v in self._data.items()]
        if self._const != 0 or not terms:
            terms.append(f"{self._const}")
        return " + ".join(terms)

    def __str__(self):
        return self.expression()

    __repr__ = __str__


PR = ParameterResolver


def to_pr(value, names=None):
    """Convert a dict / array / PR into a ParameterResolver of parameter values.

    An array is zipped against ``names`` (the circuit's parameter names), as the
    reference's ``_check_and_generate_pr_type`` does (utils/type_value_check.py).
    """
    if isinstance(value, ParameterResolver):
        return value
    if isinstance(value, dict):
        return ParameterResolver(value)
    if isinstance(value, (list, tuple, np.ndarray)):
        arr = np.asarray(value).reshape(-1)
        if names is None or len(names) != arr.size:
            raise ValueError(f"Need {0 if names is None else len(names)} parameter values, but get {arr.size}.")
        return ParameterResolver(dict(zip(names, arr.tolist())))
    if isinstance(value, numbers.Number) and names is not None and len(names) == 1:
        return ParameterResolver({names[0]: value})
    raise TypeError(f"Cannot convert {type(value)} to a parameter resolver.")


def _ordered_union(lists: Iterable[Iterable[str]]):
    out = {}
    for lst in lists:
        for k in lst:
            out.setdefault(k, None)
    return list(out.keys())
