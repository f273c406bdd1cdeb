/*
 * gsknn_ref.h -- the reference-algorithm entry points of libgsknn.so under the header name the
 * GSKNN reference uses for them (ChenhanYu/rnn, include/gsknn_ref.h: dgsknn_ref, sgsknn_ref,
 * defined in frame/gsknn_ref.c:63-162). A program written against the reference, such as its
 * test drivers test/test_dgsknn.c and test/test_sgsknn.c, includes <gsknn.h> and <gsknn_ref.h>
 * and compiles unchanged against this include directory.
 *
 * The prototypes are the ones gsknn.h already declares; this file only adds the header name.
 */
#ifndef GSKNN_B200_REF_H
#define GSKNN_B200_REF_H

#include "gsknn.h"

#endif /* GSKNN_B200_REF_H */
