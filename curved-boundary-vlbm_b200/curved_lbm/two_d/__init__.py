"""D2Q4x6 curved-boundary solver."""
