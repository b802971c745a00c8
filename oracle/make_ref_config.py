"""Write the configuration headers the reference's C++ sources include (normally generated by its
CMake build from cmake/cmake_config.h.in and cmake/lang20_config.h.in.in) into oracle/_ref/config/.

Test infrastructure for building the reference CPU simulator out of tree (oracle/Makefile, target
_ref/libmqref.so).  Values: VERSION_INFO "0.12.0", no abseil, no long double (with it,
ComplexCast<double, double> does not compile at cpu_vector_core_policy.cpp:151), every C++20
feature macro 1 except std::format and the detection TS v2, which GCC 13 lacks.

    python oracle/make_ref_config.py <reference root> <output dir>
"""
import os
import re
import sys

OFF = {'HAS_CXX20_FORMAT', 'HAS_DETECTED_TS2'}


def main(ref, out):
    os.makedirs(out, exist_ok=True)
    with open(os.path.join(out, 'cmake_config.h'), 'w', encoding='utf8') as f:
        f.write('#ifndef CMAKE_CONFIG_HPP_IN\n#define CMAKE_CONFIG_HPP_IN\n#define VERSION_INFO "0.12.0"\n'
                '#define MQ_HAS_ABSEIL_CPP 0\n#define MQ_HAS_LONG_DOUBLE 0\n#endif\n')
    with open(os.path.join(ref, 'cmake', 'lang20_config.h.in.in'), encoding='utf8') as f:
        tmpl = f.read()
    for lang, name in (('CXX', 'cxx20_config.h'), ('CUDA', 'cuda20_config.h')):
        lines = []
        for line in tmpl.replace('@LANG@', lang).splitlines():
            m = re.match(r'@MQ_DEFINE_MACRO@ (MQ_\w+)', line)
            if m:
                macro = m.group(1)
                feature = macro[len(f'MQ_{lang}_'):]
                lines.append(f'#define {macro} {0 if feature in OFF else 1}')
            else:
                lines.append(line)
        with open(os.path.join(out, name), 'w', encoding='utf8') as f:
            f.write('\n'.join(lines) + '\n')


if __name__ == '__main__':
    main(sys.argv[1], sys.argv[2])
