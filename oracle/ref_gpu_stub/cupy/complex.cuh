/* Empty stand-in for CuPy's complex header: the reference's GPU kernels
 * (blond/gpu/kernels.cu) include it but use no complex type, and CuPy is not
 * installed here.  Used only to build the reference kernels as a baseline. */
#pragma once
