"""Ready-made scheme presets (``src/gpusw/schemes.py:23-39`` of the reference package).

Look them up by attribute (``schemes.BLOSUM62``) or by name through
:meth:`Scheme.preset` / the ``scheme=`` argument of the helpers.
"""
from __future__ import annotations

from .matrix import Matrix
from .scheme import Scheme

__all__ = ["DNA", "DNA_GLOBAL", "DNA_SEMIGLOBAL", "BLASTN", "EDNAFULL", "BLOSUM62",
           "BLOSUM62_GLOBAL", "PROTEIN_SEMIGLOBAL"]

DNA = Scheme(mode="local", match=2, mismatch=-3, gap_open=-5, gap_extend=-2)
DNA_GLOBAL = DNA.replace(mode="global")
DNA_SEMIGLOBAL = DNA.replace(mode="semiglobal")
BLASTN = Scheme(mode="local", match=2, mismatch=-3, gap_open=-5, gap_extend=-2)
EDNAFULL = Scheme(mode="global", matrix=Matrix.named("EDNAFULL"), gap_open=-10, gap_extend=-1)
BLOSUM62 = Scheme(mode="local", matrix=Matrix.named("BLOSUM62"), gap_open=-11, gap_extend=-1)
BLOSUM62_GLOBAL = BLOSUM62.replace(mode="global")
PROTEIN_SEMIGLOBAL = BLOSUM62.replace(mode="semiglobal")
