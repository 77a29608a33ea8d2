#!/usr/bin/env bash
# Test infrastructure: builds the reference's own OpenMP/sequential MPM path
# (littlemine/zpc, its include/ tree at $ZSMPM_REFERENCE_ROOT, by default the directory
# "reference" beside this repository) into the executable oracle/_ref/zsref_cli,
# driven by oracle/ref_driver.cpp and oracle/ref_cli.cpp, and the check of include/zsmpm_zpc.hpp
# against zpc's containers (oracle/zpc_adapter_check, linked with libzsmpm.so).  The output is
# the checker and the CPU baseline, never the product.
#
# zpc's CMake build needs the zpc_tpls submodule, which is not checked out, so the needed
# translation units are compiled directly with g++.  Several reference headers do not parse
# with g++ 13 because a dependent member template is named without the `template`
# keyword (or call a member of a dependent base without this->), and G2P2G.hpp calls the
# CUDA-only two-argument atomicAdd; for those, patched
# copies are written under oracle/_ref/patched (searched before the reference tree).
# No patch touches arithmetic:
#   ZpcAsync.hpp                        _storage[i].data<T>()  -> .template data<T>()
#   simulation/transfer/G2P.hpp         grid_block.pack<N>()   -> .template pack<N>()
#   simulation/transfer/G2C2P.hpp       block.pack<N>()        -> .template pack<N>()
#   simulation/grid/GridOp.hpp          block.pack<N>()        -> .template pack<N>()
#   types/View.h                        dof_detail::T_t        -> dof_detail::template T_t;
#                                       typename integral_constant<..> -> integral_constant<..>
#   simulation/transfer/G2P2G.hpp       atomicAdd(&r, v) -> atomic_add(wrapv<space>{}, &r, v),
#                                       the exec-space atomic that P2G.hpp uses (a plain add
#                                       under seq_exec)
#   geometry/AnalyticLevelSet.h,        getSignedDistance(..) -> this->getSignedDistance(..)
#   geometry/SparseLevelSet.hpp         in the finite-difference normals (a member of the
#                                       CRTP base); the other geometry headers are linked beside
#                                       them so that their relative includes find the patched copies
# Logging (plog) and magic_enum are replaced by the small shims in oracle/ref_shims.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${ZSMPM_REFERENCE_ROOT:-$(cd "$HERE/../.." && pwd)/reference}/include"
OUT="$HERE/_ref"
if [ ! -d "$REF/zensim" ]; then
  echo "build_ref: reference sources not found at $REF; keeping any prebuilt $OUT" >&2
  exit 0
fi
mkdir -p "$OUT/patched/zensim/simulation/transfer" "$OUT/patched/zensim/simulation/grid" "$OUT/obj"
sed -E 's/_storage\[([^]]*)\]\.data</_storage[\1].template data</g' \
  "$REF/zensim/ZpcAsync.hpp" > "$OUT/patched/zensim/ZpcAsync.hpp"
sed -E 's/(grid_block|block)\.pack</\1.template pack</g' \
  "$REF/zensim/simulation/transfer/G2P.hpp" > "$OUT/patched/zensim/simulation/transfer/G2P.hpp"
sed -E 's/(grid_block|block)\.pack</\1.template pack</g' \
  "$REF/zensim/simulation/grid/GridOp.hpp" > "$OUT/patched/zensim/simulation/grid/GridOp.hpp"
sed -E 's/(grid_block|block)\.pack</\1.template pack</g' \
  "$REF/zensim/simulation/transfer/G2C2P.hpp" > "$OUT/patched/zensim/simulation/transfer/G2C2P.hpp"
mkdir -p "$OUT/patched/zensim/types"
sed -E -e 's/= typename integral_constant</= integral_constant</' \
  -e 's/dof_detail::(value_t|T_t|size_t|index_t|counter_t|dim_t|extent_t)/dof_detail::template \1/g' \
  "$REF/zensim/types/View.h" > "$OUT/patched/zensim/types/View.h"
sed -E 's/atomicAdd\(/atomic_add(wrapv<space>{}, /g' \
  "$REF/zensim/simulation/transfer/G2P2G.hpp" > "$OUT/patched/zensim/simulation/transfer/G2P2G.hpp"
# relative includes of the patched copies ("Scheme.hpp", "../transfer/Scheme.hpp", "Property.h")
ln -sf "$REF/zensim/simulation/transfer/Scheme.hpp" "$OUT/patched/zensim/simulation/transfer/Scheme.hpp"
ln -sf "$REF/zensim/types/Property.h" "$OUT/patched/zensim/types/Property.h"
mkdir -p "$OUT/patched/zensim/geometry"
for f in "$REF"/zensim/geometry/*; do
  case "$(basename "$f")" in
    AnalyticLevelSet.h | SparseLevelSet.hpp)
      rm -f "$OUT/patched/zensim/geometry/$(basename "$f")"
      sed -E 's/\(getSignedDistance\(/(this->getSignedDistance(/g; s/- getSignedDistance\(/- this->getSignedDistance(/g' \
        "$f" > "$OUT/patched/zensim/geometry/$(basename "$f")" ;;
    *) ln -sfn "$f" "$OUT/patched/zensim/geometry/$(basename "$f")" ;;
  esac
done

CXXFLAGS=(-std=c++17 -O2 -fPIC -fopenmp -ffp-contract=off -include cstdint -include utility
  -DZS_ENABLE_OPENMP=1 -DZS_ENABLE_CUDA=0 -DZS_ENABLE_MUSA=0 -DZS_ENABLE_SYCL=0
  -DZS_ENABLE_SYCL_ONEAPI=0 -DZS_ENABLE_SYCL_ACPP=0 -DZS_ENABLE_ROCM=0
  -DZS_ENABLE_OFB_ACCESS_CHECK=0 -DZS_ENABLE_SERIALIZATION=0 -DZS_ENABLE_VULKAN=0
  -DZS_BUILD_SHARED_LIBS=0 -DZS_ENABLE_OPENVDB=0 -DZS_ENABLE_JIT=0
  -I"$OUT/patched" -I"$HERE/ref_shims" -I"$REF")
SOURCES=(container/Vector.cpp container/TileVector.cpp container/HashTable.cpp container/Bht.cpp
  memory/Allocator.cpp memory/MemOps.cpp memory/MemoryBackend.cpp
  resource/Resource.cpp resource/ExecutionPolicy.cpp resource/omp/ExecutionPolicy.cpp
  execution/ConcurrencyPrimitive.cpp execution/ManagedThread.cpp execution/Stacktrace.cpp
  ZpcInitialization.cpp)
OBJS=()
pids=()
for s in "${SOURCES[@]}"; do
  o="$OUT/obj/$(echo "$s" | tr '/' '_' | sed 's/\.cpp$/.o/')"
  OBJS+=("$o")
  if [ ! -f "$o" ] || [ "$REF/zensim/$s" -nt "$o" ]; then
    g++ "${CXXFLAGS[@]}" -c "$REF/zensim/$s" -o "$o" &
    pids+=($!)
  fi
done
g++ "${CXXFLAGS[@]}" -c "$HERE/ref_shims/cpp_timer.cpp" -o "$OUT/obj/cpp_timer.o" &
pids+=($!)
g++ "${CXXFLAGS[@]}" -c "$HERE/ref_driver.cpp" -o "$OUT/obj/ref_driver.o" &
pids+=($!)
g++ "${CXXFLAGS[@]}" -c "$HERE/ref_cli.cpp" -o "$OUT/obj/ref_cli.o" &
pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
g++ -fopenmp -o "$OUT/zsref_cli" "$OUT/obj/ref_cli.o" "$OUT/obj/ref_driver.o" \
  "$OUT/obj/cpp_timer.o" "${OBJS[@]}" -lpthread -ldl
echo "build_ref: wrote $OUT/zsref_cli"
# the check of include/zsmpm_zpc.hpp against zpc's own containers, linked with libzsmpm.so
LIBDIR="$HERE/../zsmpm_b200/lib"
if [ -f "$LIBDIR/libzsmpm.so" ]; then
  g++ "${CXXFLAGS[@]}" -I"$HERE/../include" -c "$HERE/zpc_adapter_check.cpp" -o "$OUT/obj/zpc_adapter_check.o"
  g++ -fopenmp -o "$OUT/zpc_adapter_check" "$OUT/obj/zpc_adapter_check.o" "$OUT/obj/cpp_timer.o" "${OBJS[@]}" \
    -L"$LIBDIR" -lzsmpm -Wl,-rpath,'$ORIGIN/../../zsmpm_b200/lib' -lpthread -ldl
  echo "build_ref: wrote $OUT/zpc_adapter_check"
fi
