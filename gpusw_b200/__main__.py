"""``python -m gpusw_b200`` runs the command-line interface."""
from .cli import main

raise SystemExit(main())
