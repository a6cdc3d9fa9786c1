# Handler modules of the rtspatial_b200 library, for CMake projects.
#
#   include(<rtspatial_b200>/cmake/rtspatial_shaders.cmake)
#   RTSPATIAL_COMPILE_SHADERS(<handler include dir> <handler header> <output dir> <out var>)
#
# Same name and arguments as the reference's function (its CMakeLists.txt:73-104):
# compiles this library's handler-module source with the handler header
# force-included, for sm_100a, into <output dir>/rtspatial_handlers.cubin, and
# sets <out var> to that file.  Add it to a target's sources (as the
# reference's projects add their PTX files) so it is built before the target,
# and pass <output dir> as rtspatial::Config::ptx_root: Init loads the module
# and every query calls the header's rtspatial_handle_* functions per pair.
#
# Handler headers written for the reference include <optix.h> without using
# it; an empty stand-in is the last -I directory, so such a header compiles
# unchanged without the OptiX SDK (an optix.h in an earlier include directory
# is used instead).
get_filename_component(RTSPATIAL_B200_ROOT "${CMAKE_CURRENT_LIST_DIR}/.." ABSOLUTE)

function(RTSPATIAL_COMPILE_SHADERS CALLBACK_INCLUDE_DIR CALLBACK_HEADER OUTPUT_DIR GENERATED_FILES)
  if(CMAKE_CUDA_COMPILER)
    set(_nvcc "${CMAKE_CUDA_COMPILER}")
  else()
    find_program(_nvcc nvcc HINTS "$ENV{CUDA_HOME}/bin" /usr/local/cuda/bin REQUIRED)
  endif()
  set(_src "${RTSPATIAL_B200_ROOT}/rtspatial_b200/shaders/rts_handler_module.cu")
  set(_csrc "${RTSPATIAL_B200_ROOT}/rtspatial_b200/csrc")
  set(_out "${OUTPUT_DIR}/rtspatial_handlers.cubin")
  set(_compat "${OUTPUT_DIR}/compat")
  file(MAKE_DIRECTORY "${_compat}")
  file(WRITE "${_compat}/optix.h"
       "/* Empty: handler headers written for RTSpatial include <optix.h> but use nothing from it. */\n")
  if(IS_ABSOLUTE "${CALLBACK_HEADER}")
    set(_header_dep "${CALLBACK_HEADER}")
  else()
    set(_header_dep "${CALLBACK_INCLUDE_DIR}/${CALLBACK_HEADER}")
  endif()
  file(GLOB _deps "${_csrc}/*.cuh" "${_csrc}/*.h" "${RTSPATIAL_B200_ROOT}/include/rtspatial/*/*.h")
  add_custom_command(
    OUTPUT "${_out}"
    COMMAND "${_nvcc}" -cubin -gencode arch=compute_100a,code=sm_100a -std=c++17 -O3
            -fmad=false --expt-relaxed-constexpr
            -I "${RTSPATIAL_B200_ROOT}/include" -I "${_csrc}" -I "${CALLBACK_INCLUDE_DIR}"
            -I "${_compat}" -include "${CALLBACK_HEADER}" "${_src}" -o "${_out}"
    DEPENDS "${_src}" "${_header_dep}" ${_deps}
    COMMENT "rtspatial_b200 handler module (${CALLBACK_HEADER}) -> ${_out}"
    VERBATIM)
  set(${GENERATED_FILES} "${_out}" PARENT_SCOPE)
endfunction()
