# CMake package of tensorforge_b200 (find_package(TensorForge)), the counterpart of the
# reference's share/cmake/TensorForgeConfig.cmake: it provides
#   TensorForge_INCLUDE_DIRS  directory of tensorforge_aux.h (and the other C headers)
#   TensorForge_SOURCES       the runtime helper source generated launchers link against
#   TensorForge::TensorForge  INTERFACE target carrying both
# Generated kernels target sm_100a only, so DEVICE_BACKEND must be "cuda" (the default);
# the other backends the reference accepts are rejected with an error here.
include(FindPackageHandleStandardArgs)

get_filename_component(_tfb_pkg "${CMAKE_CURRENT_LIST_DIR}/../.." ABSOLUTE)
get_filename_component(_tfb_root "${_tfb_pkg}/.." ABSOLUTE)

find_path(TensorForge_INCLUDE_DIRS tensorforge_aux.h
          PATHS "${_tfb_pkg}/include" "${_tfb_root}/include" NO_DEFAULT_PATH)
find_file(TensorForge_SOURCES tensorforge_aux.cu
          PATHS "${_tfb_pkg}/csrc" NO_DEFAULT_PATH)

if(NOT DEFINED DEVICE_BACKEND)
  set(DEVICE_BACKEND "cuda" CACHE STRING "device backend of the generated kernels")
  set_property(CACHE DEVICE_BACKEND PROPERTY STRINGS "cuda")
elseif(NOT DEVICE_BACKEND STREQUAL "cuda")
  message(FATAL_ERROR "DEVICE_BACKEND=${DEVICE_BACKEND}: tensorforge_b200 generates CUDA for sm_100a only (use cuda)")
endif()

find_package_handle_standard_args(TensorForge
                                  REQUIRED_VARS TensorForge_INCLUDE_DIRS TensorForge_SOURCES
                                  VERSION_VAR PACKAGE_VERSION)

if(TensorForge_FOUND AND NOT TARGET TensorForge::TensorForge)
  add_library(TensorForge::TensorForge INTERFACE IMPORTED)
  set_target_properties(TensorForge::TensorForge PROPERTIES
    INTERFACE_INCLUDE_DIRECTORIES "${TensorForge_INCLUDE_DIRS}"
    INTERFACE_SOURCES "${TensorForge_SOURCES}")
  # the launchers and kernels are compiled for sm_100a only
  set(TensorForge_CUDA_ARCHITECTURES "100a")
endif()
