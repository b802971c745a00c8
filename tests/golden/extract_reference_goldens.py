"""Extract the golden numbers of the reference's own tests and docstrings into reference_goldens.json.

The reference Python package cannot be imported here (its compiled modules are not
built), so the golden vectors are read as text from the reference sources and stored
with their file:line of origin.  Run from the repository root:

    python tests/golden/extract_reference_goldens.py /root/reference

The JSON it writes is committed; the tests read only the JSON.
"""
import ast
import json
import os
import re
import sys


def _find_line(lines, pattern, start=0):
    for i in range(start, len(lines)):
        if re.search(pattern, lines[i]):
            return i
    raise LookupError(pattern)


def _literal_after(lines, start, opener):
    """Parse the python literal that starts at the first ``opener`` at/after line ``start``."""
    text = "\n".join(lines[start:])
    pos = text.index(opener)
    depth = 0
    for j in range(pos, len(text)):
        if text[j] in '([{':
            depth += 1
        elif text[j] in ')]}':
            depth -= 1
            if depth == 0:
                src = text[pos:j + 1]
                break
    src = re.sub(r'\s+', ' ', src)
    return ast.literal_eval(src)


def _cplx(v):
    if isinstance(v, list):
        return [_cplx(x) for x in v]
    v = complex(v)
    return [v.real, v.imag]


def _number_after(line, name):
    m = re.search(name + r'\s*=\s*([-+0-9.eE]+)', line)
    return float(m.group(1))


def main(ref):
    out = {}
    path = 'tests/st/test_simulator/test_simulator.py'
    lines = open(os.path.join(ref, path), encoding='utf8').read().splitlines()

    i = _find_line(lines, r'def test_all_gate_with_simulator')
    j = _find_line(lines, r'qs_exp = np.array\(', i)
    out['all_gate_qs'] = {'source': f'{path}:{j + 1}', 'pr': {'a': 1, 'b': 2, 'c': 3},
                          'qs': _cplx(_literal_after(lines, j, '['))}

    i = _find_line(lines, r'def test_multi_params_gate')
    j = _find_line(lines, r'qs_exp = np.array\(', i)
    k = _find_line(lines, r'f_exp = np.array\(', j)
    g = _find_line(lines, r'g_exp = np.array\(', k)
    out['multi_params'] = {'source': f'{path}:{j + 1}', 'p0': [1.0, 2.0, 3.0, 4.0, 5.0],
                           'qs': _cplx(_literal_after(lines, j, '[')),
                           'f': _cplx(_literal_after(lines, k, '[')),
                           'g': _cplx(_literal_after(lines, g, '['))}

    i = _find_line(lines, r'def test_custom_gate_in_parallel')
    j = _find_line(lines, r'f_sum_exp\s*=', i)
    k = _find_line(lines, r'g_sum_exp\s*=', i)
    out['custom_gate_in_parallel'] = {'source': f'{path}:{j + 1}', 'seed': 42,
                                      'f_sum': _number_after(lines[j], 'f_sum_exp'),
                                      'g_sum': _number_after(lines[k], 'g_sum_exp')}

    i = _find_line(lines, r'def test_mul_qubit_gate')
    j = _find_line(lines, r'assert np.allclose\(f1,', i)
    k = _find_line(lines, r'assert np.allclose\(g1,', i)
    out['mul_qubit_gate'] = {'source': f'{path}:{j + 1}', 'p': 2.3,
                             'f1': float(re.search(r'f1,\s*([-0-9.]+)', lines[j]).group(1)),
                             'g1': float(re.search(r'g1,\s*([-0-9.]+)', lines[k]).group(1))}

    path = 'mindquantum/simulator/simulator.py'
    lines = open(os.path.join(ref, path), encoding='utf8').read().splitlines()
    i = _find_line(lines, r"sim.apply_circuit\(Circuit\(\).ry\('a', 0\).ry\('b', 1\), np.array\(\[1.1, 2.2\]\)\)")
    amps = []
    for t in range(i + 1, i + 12):
        m = re.match(r'\s*([-0-9.e]+)¦(\d+)⟩', lines[t])
        if m:
            amps.append((int(m.group(2), 2), float(m.group(1))))
    out['apply_circuit_doc'] = {'source': f'{path}:{i + 1}', 'pr': [1.1, 2.2],
                                'qs': [[v, 0.0] for _, v in sorted(amps)]}
    i = _find_line(lines, r'grad_ops\(np.array\(\[1.0\]\)\)')
    m = re.findall(r'([-0-9.]+)\+0\.j', lines[i + 1])
    out['grad_doc'] = {'source': f'{path}:{i + 2}', 'p': 1.0, 'f': float(m[0]), 'g': float(m[1])}
    i = _find_line(lines, r"res = sim.sampling\(circ, \{'a': 1.1, 'b': 2.2\}, shots=100, seed=42\)")
    k = _find_line(lines, r"^\s*\{'[01]+': \d+", i)
    out['sampling_doc'] = {'source': f'{path}:{k + 1}', 'pr': {'a': 1.1, 'b': 2.2}, 'shots': 100, 'seed': 42,
                           'counts': ast.literal_eval(lines[k].strip())}

    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'reference_goldens.json')
    with open(dst, 'w', encoding='utf8') as f:
        json.dump(out, f, indent=1)
    print(f"wrote {dst}")


if __name__ == '__main__':
    if len(sys.argv) != 2:
        sys.exit('usage: python tests/golden/extract_reference_goldens.py <reference checkout>')
    main(sys.argv[1])
