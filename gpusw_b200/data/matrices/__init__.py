"""Bundled substitution matrices in NCBI/BLAST text format."""
