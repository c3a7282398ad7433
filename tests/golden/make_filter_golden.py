"""Generate the filter-spectrum fixtures from the reference's own genFilter
(src/Filters.cpp, built from its sources into oracle/_ref by oracle/ref.mk).

    python tests/golden/make_filter_golden.py

Writes tests/golden/filters_reference.npz: for every spectral filter type
(ram-lak .. parzen), FFT sizes N in SIZES, cut-offs d in DS and, for the types
that take one, a non-default parameter, the reference's spectrum on bins
0 .. N/2.  Keys '<name>|<N>|<d>|<parameter>'.  Host code only: runs without a
GPU.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

SIZES = (128, 256, 2048)
DS = (1.0, 0.7)
PARAMS = {'tukey': 0.3, 'gaussian': 0.25, 'blackman': 0.2, 'kaiser': 2.0}
NAMES = ['ram-lak', 'shepp-logan', 'cosine', 'hamming', 'hann', 'tukey', 'lanczos', 'triangular', 'gaussian',
         'barlett-hann', 'blackman', 'nuttall', 'blackman-harris', 'blackman-nuttall', 'flat-top', 'kaiser',
         'parzen']


def main():
    from oracle import ref
    out = {}
    for name in NAMES:
        ref_type = NAMES.index(name) + 2  # FILTER_ERROR, FILTER_NONE come first in E_FBPFILTER
        for N in SIZES:
            for d in DS:
                for p in (-1.0, PARAMS.get(name)):
                    if p is None:
                        continue
                    out['%s|%d|%g|%g' % (name, N, d, p)] = ref.gen_filter(ref_type, N, d, p)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'filters_reference.npz')
    np.savez_compressed(path, **out)
    print("wrote %d spectra to %s" % (len(out), path))


if __name__ == '__main__':
    main()
