"""Trained rank model of the learned-rank sparsification (rank_mlp.npz) and
the script that produced it (train_rank_model.py)."""
