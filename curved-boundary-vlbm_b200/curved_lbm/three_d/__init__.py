"""D3Q6x12 sparse curved-boundary solver."""
