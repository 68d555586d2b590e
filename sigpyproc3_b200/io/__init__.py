"""Filterbank file I/O: sigproc headers, bit layouts and the streaming reader."""
