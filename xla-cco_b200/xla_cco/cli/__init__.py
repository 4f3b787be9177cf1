"""Command-line drivers (``python -m xla_cco.cli.relax``)."""
