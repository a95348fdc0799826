// Empty stand-in for <hpx/async.hpp>: the reference's 1D FFT sources include
// it but call nothing from it.
#pragma once
