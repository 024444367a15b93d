"""B200 CBS3D step engine: case generator and the Python host over the C ABI."""
