"""I/O dataset protocols (same interface as the reference's cuphu.io)."""
from cuphu_b200.io._dataset import InputDataset, OutputDataset

__all__ = ["InputDataset", "OutputDataset"]
