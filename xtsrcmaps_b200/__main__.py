"""Command line: the reference's main.cxx flow for point sources, end to end.

    python -m xtsrcmaps_b200 --config c1 --out srcmaps.fits

main.cxx:17-40 collects the configuration, observation, sources and IRFs, runs
compute_exposure, compute_psf_data and compute_srcmaps (:28-30) and would write
the maps with fits::write_src_model (:40, commented out there).  Every input
starts as the seeded synthetic job of the named configuration and can be
replaced by the reference's own files: --ccube (counts cube: WCS and energies,
observation/observation.cxx), --ltcube (livetime cube, EXPOSURE and
WEIGHTED_EXPOSURE tables), --aeff and --psf (Pass-8 IRF files), --xml (point
sources of a source model), or --sources (an .npz with ``src_sph`` [S, 2] degrees
and ``names``).  The three calls run as one device call and the maps go to the
FITS file from device memory.  --adaptive RTOL uses the adaptive cubature, and
--surrogate / --train-surrogate the learned surrogate of the pixel cubature (with
the 12-point rule where it does not apply).
"""
from __future__ import annotations

import argparse
import sys
import time


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m xtsrcmaps_b200", description=__doc__.splitlines()[0])
    ap.add_argument("--config", default="c1", choices=["c0", "c1", "c2", "c4"], help="synthetic job")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--sources", help=".npz with src_sph [S, 2] (deg) and optional names")
    ap.add_argument("--xml", help="source model XML: its point sources")
    ap.add_argument("--ccube", help="counts cube FITS: map WCS and energies")
    ap.add_argument("--ltcube", help="livetime cube FITS (EXPOSURE, WEIGHTED_EXPOSURE tables)")
    ap.add_argument("--aeff", help="effective-area IRF FITS (EFFECTIVE AREA_*, EFFICIENCY_PARAMS_*)")
    ap.add_argument("--psf", help="PSF IRF FITS (RPSF_*, PSF_SCALING_PARAMS_*)")
    ap.add_argument("--out", required=True, help="output FITS file")
    ap.add_argument("--bitpix", type=int, default=-64, choices=[-64, -32])
    ap.add_argument("--adaptive", type=float, default=None, metavar="RTOL",
                    help="adaptive Genz-Malik cubature at this relative tolerance instead of the 12-point rule")
    ap.add_argument("--surrogate", metavar="NET.npz", help="pixel means from this trained surrogate network "
                    "(the 12-point rule where it does not apply)")
    ap.add_argument("--train-surrogate", metavar="NET.npz", help="train a surrogate network on samples of this "
                    "job's mean PSFs, save it here and use it")
    ap.add_argument("--surrogate-samples", type=int, default=10_000_000)
    ap.add_argument("--surrogate-epochs", type=int, default=60)
    ap.add_argument("--check-tol", type=float, default=1e-4,
                    help="surrogate maps whose check against the rule exceeds this are redone by the rule")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)

    import numpy as np
    import torch

    from . import api as A
    from . import fits_io, irf
    from .synth import make_job

    job = make_job(args.config, seed=args.seed)
    names = list(job.src_names) if job.src_names else ["SRC%05d" % s for s in range(job.S)]
    if args.sources:
        z = np.load(args.sources, allow_pickle=False)
        job.src_sph = np.ascontiguousarray(z["src_sph"], dtype=np.float64)
        names = [str(n) for n in z["names"]] if "names" in z.files else ["SRC%05d" % s for s in range(job.S)]
    if args.xml:
        from .sources import read_point_sources

        names, job.src_sph = read_point_sources(args.xml)
    if args.ccube:  # observation/observation.cxx: WCS from the cube, energies from EBOUNDS
        job.wcs, _ = fits_io.read_image_meta(args.ccube)
        job.energies = fits_io.read_energies(args.ccube)
        job.logEs = np.log10(job.energies)
    if args.ltcube:
        job.exp_cube = fits_io.read_expcube(args.ltcube, "EXPOSURE")
        job.wexp_cube = fits_io.read_expcube(args.ltcube, "WEIGHTED_EXPOSURE")
    if args.aeff:
        a = irf.load_aeff(args.aeff)
        job.aeff_front, job.aeff_back = a["front"].grid, a["back"].grid
        job.effic_front = a["front"].effic
    if args.psf:
        p = irf.load_psf(args.psf)
        job.rpsf_front, job.rpsf_back = p["front"].grid, p["back"].grid
        job.scale_front, job.scale_back = p["front"].scale, p["back"].scale
    A.init(args.device)
    dev = torch.device("cuda", args.device)
    t0 = time.perf_counter()
    ltf = A.livetime_efficiency_factors(job.logEs, job.effic_front)
    nf = A.normalize_rpsf(job.rpsf_front, job.scale_front)
    nb = A.normalize_rpsf(job.rpsf_back, job.scale_back)
    src = torch.as_tensor(job.src_sph, device=dev)
    use_sur = args.surrogate or args.train_surrogate
    if args.adaptive is not None and use_sur:
        ap.error("--adaptive and the surrogate options exclude each other")
    if args.adaptive is None and not use_sur:
        cube = A.ExpCube(torch.as_tensor(job.exp_cube.cosbins, device=dev), job.exp_cube.nside,
                         job.exp_cube.nbrbins, job.exp_cube.cosmin, job.exp_cube.thetabin)
        wcube = A.ExpCube(torch.as_tensor(job.wexp_cube.cosbins, device=dev), job.wexp_cube.nside,
                          job.wexp_cube.nbrbins, job.wexp_cube.cosmin, job.wexp_cube.thetabin)
        maps, _ = A.point_source_maps(job.wcs, src, cube, wcube, torch.as_tensor(job.logEs, device=dev),
                                      job.aeff_front, job.aeff_back, nf, nb, torch.as_tensor(ltf, device=dev),
                                      with_info=False)
    else:
        ex = A.compute_exposure(job.exp_cube, job.wexp_cube, job.logEs, job.src_sph, job.aeff_front,
                                job.aeff_back, ltf)
        ps = A.compute_psf_data(nf, nb, ex, job.logEs, ltf)
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
        if args.adaptive is not None:
            maps, _ = A.point_src_model_map_wcs_adaptive(job.wcs, src, t(ex.exposure), t(ps.uPsf),
                                                         t(ps.partial_psf_integral), rtol=args.adaptive,
                                                         with_info=False)
        else:
            from .surrogate import Surrogate, samples

            if args.train_surrogate:
                X, Y = samples(t(ps.uPsf), job.logEs, args.surrogate_samples, seed=args.seed)
                net = Surrogate(device=dev, seed=args.seed)
                losses = net.train(X, Y, epochs=args.surrogate_epochs)
                del X, Y
                # error cells from held-out samples of the same tables (another seed)
                Xc, Yc = samples(t(ps.uPsf), job.logEs, max(1_000_000, args.surrogate_samples // 3),
                                 seed=args.seed + 1)
                cal = net.calibrate(Xc, Yc, tol=args.check_tol, margin=0.7)
                del Xc, Yc
                print(f"surrogate calibrated: {cal['cells_accepted']} of {cal['cells']} cells served, "
                      f"{cal['share_in_accepted_cells']:.3f} of held-out samples in them")
                net.save(args.train_surrogate)
                print(f"surrogate trained: {args.surrogate_samples} samples, {args.surrogate_epochs} epochs, "
                      f"loss {losses[0]:.3e} -> {losses[-1]:.3e}, saved to {args.train_surrogate}")
            else:
                net = Surrogate.load(args.surrogate, device=dev)
            maps, _, st = A.point_src_model_map_wcs_surrogate(job.wcs, src, t(ex.exposure), t(ps.uPsf),
                                                              t(ps.partial_psf_integral), t(job.logEs), net,
                                                              check_tol=args.check_tol, with_info=False)
            print(f"surrogate: {st['accepted']} of {st['values']} values from the network, "
                  f"{st['maps_fallback']} maps redone by the rule (largest check difference "
                  f"{st['max_check_err']:.2e})")
    t1 = time.perf_counter()
    A.write_src_model(args.out, maps, names, args.bitpix)
    torch.cuda.synchronize(dev)
    t2 = time.perf_counter()
    S, H, W, E = maps.shape
    print(f"{S} sources x {H}x{W} x {E} energies: maps {t1 - t0:.3f} s, FITS {t2 - t1:.3f} s -> {args.out}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
