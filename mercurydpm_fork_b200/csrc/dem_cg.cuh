// dem_cg.cuh -- Gaussian coarse-graining (CG<Coordinates, Gauss, StandardFields>).
#pragma once

extern "C" int dem_cg_eval(dem_handle* hh, const dem_cg_grid* grid, double* fields_out)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    (void)grid;
    (void)fields_out;
    return fail(h, DEM_ERR_STATE, "dem_cg_eval: coarse-graining is not available in this build");
}
