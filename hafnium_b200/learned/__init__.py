"""The learned initial density (north-star form 4): a message-passing network over
the waters of a cluster that predicts the density matrix in each water's own frame."""
