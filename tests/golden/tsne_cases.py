"""optimize_tsne option variants (magnet/tsne.py:132-135) run on tsne_small.npz's graph and start: heavy tails
(dof 0.7), 5 interpolation points per box over wider boxes, late exaggeration with a higher late momentum. Shared
by the fixture script and the tests."""
TSNE_VARIANTS = {"dof07": dict(dof=0.7), "interp5": dict(n_interp=5, box_width=1.0),
                 "exag": dict(exaggeration=1.5, momentum=(0.5, 0.9))}
