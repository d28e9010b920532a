# Source to use the B200 libqcs.so: puts lib/ on LD_LIBRARY_PATH and the
# public headers on CPATH (same role as the reference's env.bash).
_qcs_pkg_dir="$(dirname "$(realpath "${BASH_SOURCE[0]}")")"
export LD_LIBRARY_PATH="${LD_LIBRARY_PATH:+${LD_LIBRARY_PATH}:}${_qcs_pkg_dir}/lib"
export CPATH="${CPATH:+${CPATH}:}$(dirname "${_qcs_pkg_dir}")/include"
unset _qcs_pkg_dir
