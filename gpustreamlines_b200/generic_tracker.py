"""Chunked seed loop and writers (``cuslines/generic_tracker.py:13-172``).

``generate_sft`` returns a voxel-space ``StatefulTractogram``;
``generate_trx`` streams each chunk into a memory-mapped ``TrxFile`` in RAS mm
with the reference's size guesses (2 streamlines per seed, 100 points per
streamline) and doubling resize.  ``generate_streamlines`` is an alias of
``generate_sft`` (the name some callers use); both reference names stay.
"""

from __future__ import annotations

import logging

import numpy as np

from .io import ArraySequence, Space, StatefulTractogram, Tractogram, TrxFile

logger = logging.getLogger("GPUStreamlines")


class GenericTracker:
    def __enter__(self):
        return self

    def __exit__(self, exc_type, exc, tb):
        return False

    def set_compression_parameters(self, pos_dtype=np.float32, linearize=False, tol_error=0.1,
                                   max_segment_length=10):
        """Compression of generated streamlines (TRX only).

        pos_dtype: dtype of the stored positions.  linearize: apply the
        linearisation of Presseau et al. 2015 with ``tol_error`` mm and
        ``max_segment_length`` mm.
        """
        self.pos_dtype = pos_dtype
        self.linearize = linearize
        self.tol_error = tol_error
        self.max_segment_length = max_segment_length

    def _ngpus(self):
        return getattr(self, "ngpus", 1)

    def _pos_dtype(self):
        return getattr(self, "pos_dtype", np.float32)

    def _linearize(self):
        return getattr(self, "linearize", False)

    def _tol_error(self):
        return getattr(self, "tol_error", 0.1)

    def _max_segment_length(self):
        return getattr(self, "max_segment_length", 10)

    def _divide_chunks(self, seeds):
        global_chunk_sz = self.chunk_size * self._ngpus()
        nchunks = (seeds.shape[0] + global_chunk_sz - 1) // global_chunk_sz
        return global_chunk_sz, nchunks

    def generate_sft(self, seeds, ref_img):
        seeds = np.asarray(seeds)
        global_chunk_sz, nchunks = self._divide_chunks(seeds)
        datas, lens = [], []
        for idx in range(nchunks):
            self.seed_propagator.propagate(seeds[idx * global_chunk_sz:(idx + 1) * global_chunk_sz])
            a = self.seed_propagator.as_array_sequence()
            if len(a):
                datas.append(a._data)
                lens.append(a._lengths)
        if datas:
            seq = ArraySequence.from_flat(np.concatenate(datas), np.concatenate(lens))
        else:
            seq = ArraySequence()
        return StatefulTractogram(seq, ref_img, Space.VOX)

    generate_streamlines = generate_sft

    def generate_trx(self, seeds, ref_img):
        seeds = np.asarray(seeds)
        global_chunk_sz, nchunks = self._divide_chunks(seeds)
        sl_len_guess = 100
        sl_per_seed_guess = 2
        n_sls_guess = sl_per_seed_guess * seeds.shape[0]
        trx_reference = TrxFile(reference=ref_img, pos_dtype=self._pos_dtype())
        trx_file = TrxFile(nb_streamlines=n_sls_guess, nb_vertices=n_sls_guess * sl_len_guess,
                           init_as=trx_reference)
        trx_reference.close()
        for idx in range(int(nchunks)):
            chunk = seeds[idx * global_chunk_sz:(idx + 1) * global_chunk_sz]
            if self._linearize():
                # world transform and linearisation on the device; only the
                # compressed points come back (the reference does both on the host)
                self.seed_propagator.propagate_compressed(chunk, trx_file.header["VOXEL_TO_RASMM"],
                                                          self._tol_error(), self._max_segment_length())
                sls = self.seed_propagator.as_compressed_sequence()
                if len(sls) == 0:
                    continue
            else:
                self.seed_propagator.propagate(chunk)
                tractogram = Tractogram(self.seed_propagator.as_array_sequence(),
                                        affine_to_rasmm=trx_file.header["VOXEL_TO_RASMM"])
                if len(tractogram) == 0:
                    continue
                tractogram.to_world()
                sls = tractogram.streamlines
            before = trx_file.header["NB_STREAMLINES"]
            trx_file.append_block(np.asarray(sls._data, dtype=self._pos_dtype()), sls._lengths)
            if trx_file.header["NB_STREAMLINES"] != before:
                logger.info("TRX resizing...")
        trx_file.resize()
        return trx_file
