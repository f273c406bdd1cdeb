/*
 * gsknn_ref_stl.hpp -- the STL-heap oracle entry points of libgsknn.so under the reference's
 * header name (ChenhanYu/rnn, include/gsknn_ref_stl.hpp: dgsknn_ref_stl, sgsknn_ref_stl,
 * defined in frame/gsknn_ref_stl.cpp:81-214).
 *
 * The declarations come from gsknn.h, inside extern "C", so a C++ caller links against the C
 * symbols of libgsknn.so whether or not it wraps the include in extern "C" itself (the
 * reference's test/test_sgsknn_stl.cpp and test/test_dgsknn_stl.cpp do wrap it).
 */
#ifndef GSKNN_B200_REF_STL_HPP
#define GSKNN_B200_REF_STL_HPP

#include "gsknn.h"

#endif /* GSKNN_B200_REF_STL_HPP */
