"""The stage layer (nbg_filter_*, nbg_pipeline_*): the reference stages'
options, defaults, dimensions, prepared() checks and per-row messages, on
the CPU (no call here touches a GPU).  Texts follow
filters/NormalFilter.cpp:85-160, filters/EigenvaluesFilter.cpp:77-172,
filters/CovarianceFeaturesFilter.cpp:71-262, pdal/private/MathUtils.cpp:572-611
and pdal/util/ProgramArgs.hpp:415-435."""
import numpy as np
import pytest

from gpupdal_b200 import abi
from gpupdal_b200.stages import Filter, StageError, parse_pipeline


def _ex(rows):
    return np.array(rows, dtype=[("point_id", np.uint32), ("stage", np.uint8), ("code", np.uint8)])


def test_normal_defaults_and_dims():
    f = Filter("filters.normal")
    o, rc = f.options()
    assert rc == abi.NBG_OK
    assert (o.kind, o.knn, o.always_up, o.has_viewpoint, o.refine) == (abi.STAGE_NORMAL, 8, 1, 0, 0)
    assert f.dims() == ["NormalX", "NormalY", "NormalZ", "Curvature"]
    assert f.log() == []


@pytest.mark.parametrize("vp", ["POINT(1 2 3)", "POINT Z (1 2 3)",
                                '{"type": "Point", "coordinates": [1, 2, 3]}',
                                {"type": "Point", "coordinates": [1, 2, 3]}])
def test_normal_viewpoint_forms_disable_always_up(vp):
    f = Filter("filters.normal", {"viewpoint": vp, "knn": "16"})
    o, _ = f.options()
    assert list(o.viewpoint) == [1.0, 2.0, 3.0] and o.has_viewpoint == 1 and o.always_up == 0
    assert o.knn == 16
    assert f.log() == ["Viewpoint provided. Ignoring always_up = TRUE."]


def test_normal_knn_and_radius_conflict():
    with pytest.raises(StageError, match=r"^filters\.normal: Cannot set both knn and radius\.$"):
        Filter("filters.normal", {"knn": 8, "radius": 1.0})
    f = Filter("filters.normal", {"radius": 1.0})
    o, rc = f.options()
    assert rc == abi.NBG_OK and o.use_radius == 1 and o.radius == 1.0


def test_value_errors_as_programargs():
    with pytest.raises(StageError, match=r"Invalid value 'eight' for argument 'knn'\."):
        Filter("filters.normal", {"knn": "eight"})
    with pytest.raises(StageError, match=r"Invalid value 'maybe' for argument 'always_up'\."):
        Filter("filters.normal", {"always_up": "maybe"})
    with pytest.raises(StageError, match=r"Unexpected argument 'k'\."):
        Filter("filters.eigenvalues", {"k": 8})


def test_eigenvalues_prepared_logs():
    f = Filter("filters.eigenvalues", {"normalize": True})
    o, rc = f.options()
    assert (o.kind, o.knn, o.normalize, rc) == (abi.STAGE_EIGENVALUES, 8, 1, abi.NBG_OK)
    assert f.log() == ["No radius specified. Proceeding with knn and stride, but ignoring min_k."]
    assert f.dims() == ["Eigenvalue0", "Eigenvalue1", "Eigenvalue2"]
    f = Filter("filters.eigenvalues", {"radius": -1})
    assert f.log() == ["Radius has been set. Ignoring knn and stride values.",
                       "Radius must be greater than 0."]
    f = Filter("filters.eigenvalues", {"radius": 2.5, "min_k": 6, "stride": 3})
    o, rc = f.options()
    assert rc == abi.NBG_OK and (o.use_radius, o.radius, o.min_k) == (1, 2.5, 6)
    assert Filter("filters.eigenvalues", {"stride": 2}).options()[1] == abi.NBG_OK
    assert Filter("filters.eigenvalues", {"stride": 8, "knn": 8}).options()[1] == abi.NBG_ERR_UNSUPPORTED


def test_covariancefeatures_feature_sets_and_mode():
    f = Filter("filters.covariancefeatures")
    o, _ = f.options()
    assert (o.knn, o.mode, o.feature_mask) == (10, abi.MODE_SQRT, abi.FEAT_DIMENSIONALITY)
    assert f.dims() == ["Linearity", "Planarity", "Scattering", "Verticality"]
    f = Filter("filters.covariancefeatures", {"feature_set": ["  OmniVariance", "linearity"],
                                              "mode": "RAW"})
    o, _ = f.options()
    assert o.mode == abi.MODE_RAW and f.dims() == ["Linearity", "Omnivariance"]
    f = Filter("filters.covariancefeatures", {"feature_set": "all"}, True, True)
    assert len(f.dims()) == 11 and f.dims()[-1] == "Density"
    with pytest.raises(StageError, match=r"Invalid value 'log' for argument 'mode'\."):
        Filter("filters.covariancefeatures", {"mode": "log"})


def test_covariancefeatures_prepared_checks():
    with pytest.raises(StageError, match="Density feature requires OptimalKNN and OptimalRadius "
                                         "dimensions, which are missing in the input PointView."):
        Filter("filters.covariancefeatures", {"feature_set": "density"}, True, False)
    with pytest.raises(StageError, match="Missing OptimalKNN dimension in input PointView."):
        Filter("filters.covariancefeatures", {"optimized": True})
    f = Filter("filters.covariancefeatures", {"optimized": True}, True, False)
    o, rc = f.options()
    assert rc == abi.NBG_OK and o.optimized == 1


def test_row_reports():
    f = Filter("filters.normal")
    f.report(_ex([(7, 0, abi.ROW_ZERO_COV), (3, 0, abi.ROW_TOO_FEW), (5, 1, abi.ROW_TOO_FEW)]), 0)
    assert f.log() == [
        "Skipping point 3: Not enough neighbors to compute normal.",
        "Skipping point 7: Covariance matrix is all zeros. This suggests a large number of "
        "redundant points."]
    g = Filter("filters.eigenvalues")
    g.report(_ex([(4, 0, abi.ROW_ZERO_COV)]))
    assert g.log()[-1] == ("Skipping point 4. Covariance matrix is all zeros. This suggests a "
                           "large number of redundant points. Consider using filters.sample with "
                           "a small radius to remove redundant points.")
    with pytest.raises(StageError, match=r"^filters\.eigenvalues: Cannot perform eigen decomposition\.$"):
        g.report(_ex([(9, 0, abi.ROW_EIGEN_FAIL)]))
    h = Filter("filters.covariancefeatures")
    with pytest.raises(StageError, match="Eigenvalues are all 0. Can't compute local features."):
        h.report(_ex([(2, 0, abi.ROW_ZERO_LAMBDA)]))


def test_pipeline_json_forms():
    text = ('{"pipeline": ["in.las", {"type": "filters.normal", "knn": 16}, '
            '{"type": "filters.covariancefeatures", "feature_set": "all", "threads": 8}, '
            '{"type": "writers.las", "filename": "out.las"}]}')
    st = parse_pipeline(text)
    assert [t for t, _ in st] == ["file", "filters.normal", "filters.covariancefeatures", "writers.las"]
    assert st[1][1]["knn"] == 16 and st[2][1]["threads"] == 8
    assert [t for t, _ in parse_pipeline('[{"type": "filters.eigenvalues"}]')] == ["filters.eigenvalues"]
    with pytest.raises(StageError):
        parse_pipeline('{"stages": []}')
    with pytest.raises(StageError):
        parse_pipeline('[{"type": "filters.normal",]')


def test_radius_few_report():
    f = Filter("filters.covariancefeatures", {"radius": 1.0, "min_k": 7})
    f.report(_ex([(12, 0, abi.ROW_RADIUS_FEW)]))
    assert f.log()[-1] == "Skipping point 12. Found 0 neighbors but required 7."


def test_consumer_defaults_and_dims():
    # the other consumers' addArgs defaults and addDimensions
    want = {
        "filters.approximatecoplanar": (abi.STAGE_APPROXIMATECOPLANAR, 8, ["Coplanar"]),
        "filters.estimaterank": (abi.STAGE_ESTIMATERANK, 8, ["Rank"]),
        "filters.nndistance": (abi.STAGE_NNDISTANCE, 10, ["NNDistance"]),
        "filters.optimalneighborhood": (abi.STAGE_OPTIMALNEIGHBORHOOD, 14,
                                        ["OptimalKNN", "OptimalRadius"]),
        "filters.lof": (abi.STAGE_LOF, 10, ["NNDistance", "LocalReachabilityDistance",
                                            "LocalOutlierFactor"]),
        "filters.outlier": (abi.STAGE_OUTLIER, 8, ["Classification"]),
    }
    for t, (kind, knn, dims) in want.items():
        f = Filter(t)
        o, rc = f.options()
        assert rc == abi.NBG_OK and o.kind == kind and o.knn == knn, t
        assert f.dims() == dims
        assert abi.stage_dims(o) == dims
    o, _ = Filter("filters.approximatecoplanar").options()
    assert (o.thresh1, o.thresh2) == (25.0, 6.0)
    o, _ = Filter("filters.estimaterank").options()
    assert o.thresh1 == 0.01
    o, _ = Filter("filters.optimalneighborhood").options()
    assert o.min_k == 10
    o, _ = Filter("filters.outlier").options()
    assert (o.mode, o.min_k, o.radius, o.thresh1, o.label) == (0, 2, 1.0, 2.0, 7)


def test_consumer_options():
    o, _ = Filter("filters.nndistance", {"mode": "AVG", "k": 6}).options()
    assert (o.mode, o.knn) == (1, 6)
    with pytest.raises(StageError, match="Invalid value 'median' for argument 'mode'"):
        Filter("filters.nndistance", {"mode": "median"})
    o, _ = Filter("filters.outlier", {"method": "Radius", "radius": 1.5, "min_k": -1,
                                      "class": 18}).options()
    assert (o.mode, o.radius, o.min_k, o.label) == (1, 1.5, -1, 18)
    f = Filter("filters.outlier", {"method": "sideways"})
    o, _ = f.options()
    assert o.mode == 2
    assert f.log() == ['Requested method is unrecognized. Please choose from "statistical" or '
                       '"radius".']
    o, _ = Filter("filters.optimalneighborhood", {"min_k": 4, "max_k": 9}).options()
    assert (o.min_k, o.knn) == (4, 9)
    with pytest.raises(StageError, match="Unexpected argument 'knn'"):
        Filter("filters.lof", {"knn": 4})


def test_outlier_outcome_warnings():
    for outl, inl, line in [(10, 0, "Requested filter would remove all points. Try a larger "
                                    "radius/smaller minimum neighbors."),
                            (0, 10, "Filtered cloud has no outliers!")]:
        f = Filter("filters.outlier")
        s = abi.RunStats()
        s.outliers, s.inliers = outl, inl
        f.outcome(s)
        assert f.log() == [line]
    f = Filter("filters.outlier")
    s = abi.RunStats()
    s.outliers, s.inliers = 3, 7
    f.outcome(s)
    assert f.log() == []


def test_consumer_row_reports():
    f = Filter("filters.approximatecoplanar")
    f.report(_ex([(4, 0, abi.ROW_ZERO_COV)]))
    assert f.log()[-1].startswith("Skipping point 4. Covariance matrix is all zeros.")
    with pytest.raises(StageError, match=r"^filters\.approximatecoplanar: Cannot perform eigen"):
        f.report(_ex([(1, 0, abi.ROW_EIGEN_FAIL)]))
    g = Filter("filters.optimalneighborhood")
    with pytest.raises(StageError, match="Cannot perform eigen decomposition."):
        g.report(_ex([(2, 0, abi.ROW_EIGEN_FAIL)]))
