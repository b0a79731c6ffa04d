"""Saving and loading of domains (phiPICT's phipict.io)."""
from .domain_io import load_domain, save_domain

__all__ = ["load_domain", "save_domain"]
