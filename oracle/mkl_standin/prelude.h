/*
 * prelude.h -- force-included (g++ -include) ahead of the reference sources.
 * The reference's definitionsHODLR.h uses alloc_arr<T>() before
 * definitions.h defines it, which the Intel compiler accepted; g++ needs the
 * template declared first.  This is the same declaration, nothing more.
 */
#pragma once
template <typename T> T *alloc_arr(long long int n);
