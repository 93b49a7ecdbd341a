# pose_b200.cmake — provide the target `pose_common_cuda` from libpose_b200.so.
#
# For the reference's build (common/CMakeLists.txt): when
# POSE_GPU_LABEL_STRATEGY is "b200", include this file instead of building the
# reference's pose_common_cuda static library.  The exported C ABI is the one
# of common/include/gpu_label.h, so consumers such as disk-wipe-bench link
# unchanged.  Requires nvcc for sm_100a (B200).
set(POSE_B200_DIR "${CMAKE_CURRENT_LIST_DIR}/..")
get_filename_component(POSE_B200_DIR "${POSE_B200_DIR}" ABSOLUTE)
set(POSE_B200_LIB "${POSE_B200_DIR}/libpose_b200.so")

add_custom_command(
    OUTPUT "${POSE_B200_LIB}"
    COMMAND make -C "${POSE_B200_DIR}" libpose_b200.so
    COMMENT "Building libpose_b200.so (sm_100a)"
    VERBATIM)
add_custom_target(pose_b200_build ALL DEPENDS "${POSE_B200_LIB}")

add_library(pose_common_cuda SHARED IMPORTED GLOBAL)
set_target_properties(pose_common_cuda PROPERTIES
    IMPORTED_LOCATION "${POSE_B200_LIB}"
    IMPORTED_NO_SONAME TRUE)
add_dependencies(pose_common_cuda pose_b200_build)
if(TARGET pose_common)
    set_property(TARGET pose_common_cuda APPEND PROPERTY INTERFACE_LINK_LIBRARIES pose_common)
endif()
